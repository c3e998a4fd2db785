"""Split-precision (BF16 slices on tcgen05 + FP64 refinement) solve through
the C-ABI against the FP64 path and the oracle.

Tolerances: Dirichlet fields 1e-12 relative to the oracle (the refined
result converges to the reference's discrete solution); Neumann fields the
same FP64-noise bound as the plain FP64 path with its own operators
(test_gpu_solve.TOL_NEU), see the discussion there."""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-12
TOL_NEU = 2e-10


def rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


def _cmp_neumann(sol, ref, xalp, tol):
    for k in range(sol.shape[2]):
        a, b = sol[:, :, k], ref[:, :, k]
        if abs(xalp[k]) < 1e-5:
            a, b = a - a.mean(), b - b.mean()
        assert rel(a, b) < tol, (k, rel(a, b))


@pytest.mark.parametrize("m", [17, 33, 65, 129])
def test_mixed_matches_oracle(gpu_ctx, oracle, m):
    nm = 4
    ops = oracle.Ops(m)
    gpu_ctx.pseudomat(m)
    rhs = synth.chebyshev_rhs(m, m, nm, seed=100 + m, ib=0)
    xalp = np.array([0.0, 0.5, 3.0, 31.5])
    for lam in (4.0e6, 1.0):
        ref, _ = oracle.helm3d(rhs, ops, "d", lam, xalp)
        sol = gpu_ctx.helm3d(rhs.copy(order="F"), "d", lam, xalp, precision=D.PREC_MIXED)
        assert rel(sol, ref) < TOL, lam
        assert np.all(sol[:, :, 0].imag == 0)
    ref, _ = oracle.helm3d(rhs, ops, "n", 0.0, xalp)
    sol = gpu_ctx.helm3d(rhs.copy(order="F"), "n", 0.0, xalp, precision=D.PREC_MIXED)
    _cmp_neumann(sol, ref, xalp, TOL_NEU)


def test_mixed_equals_fp64_path(gpu_ctx):
    """Same GPU operators: the refined split solve reproduces the FP64 DMMA
    solve of the same context to FP64 accuracy."""
    m, nm = 129, 8
    gpu_ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nm)
    for bound, lam in (("d", 4.0e6), ("n", 0.0)):
        rhs = synth.chebyshev_rhs(m, m, nm, seed=7, ib=0)
        a = gpu_ctx.helm3d(rhs.copy(order="F"), bound, lam, xalp, precision=D.PREC_FP64)
        b = gpu_ctx.helm3d(rhs.copy(order="F"), bound, lam, xalp, precision=D.PREC_MIXED)
        if bound == "d":
            assert rel(b, a) < TOL
        else:
            _cmp_neumann(b, a, xalp, TOL_NEU)


def test_mixed_batched_fields(gpu_ctx):
    m, nm = 65, 6
    gpu_ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nm)
    fields, singles = [], []
    for bound, lam, seed in (("d", 4.0e6, 1), ("d", 4.0e6, 2), ("d", 4.0e6, 3), ("n", 0.0, 4)):
        rhs = synth.chebyshev_rhs(m, m, nm, seed=seed, ib=0)
        singles.append(gpu_ctx.helm3d(rhs.copy(order="F"), bound, lam, xalp, precision=D.PREC_MIXED))
        r = gpu_ctx.device_array(rhs.shape)
        s = gpu_ctx.device_array(rhs.shape)
        r.upload(rhs)
        fields.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, bound=bound))
    gpu_ctx.solve_fields_dev(fields, precision=D.PREC_MIXED)
    gpu_ctx.synchronize()
    for f, ref in zip(fields, singles):
        assert np.array_equal(f["sol"].download(), ref)
        f["rhs"].free()
        f["sol"].free()


def test_mixed_rejects_large_grid(gpu_ctx):
    gpu_ctx.pseudomat(145)
    rhs = synth.chebyshev_rhs(145, 145, 1)
    with pytest.raises(D.DuctGPUError) as e:
        gpu_ctx.helm3d(rhs, "d", 1.0, [0.0], precision=D.PREC_MIXED)
    assert e.value.code == D.EARG
