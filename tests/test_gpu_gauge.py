"""The kx=0 Neumann gauge point and imported (host LAPACK) operators.

The reference pins U(iofzero+1, iofzero+1) = 0 for the singular pressure
mode (src/solvediag.f90:195-206), iofzero being the position of the smallest
|eigenvalue| in its host dgeev's output order (src/pseudomat.f90:141-152).
Two routes give the reference's point:

* the library's own eigen-decomposition with the caller's iofzero
  (ductgpu_set_gauge_point): the kx=0 field then equals the oracle's with no
  constant removed, to the Neumann tolerance of two independent FP64
  eigen-decompositions (TOL_NEU, see test_gpu_solve.py);
* the host's own operators imported on a grid-only set-up
  (ductgpu_pseudomat_ex + ductgpu_set_operators): the solve restates the
  reference arithmetic on the full passes (TOL_KERNEL).
"""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu
TOL_KERNEL = 1e-13
TOL_NEU = 2e-10


def rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


def test_grid_only_setup_needs_both_bounds(gpu_ctx, oracle):
    m = 17
    ops = oracle.Ops(m)
    gpu_ctx.pseudomat_ex(m)
    rhs = synth.chebyshev_rhs(m, m, 2, seed=3, ib=0)
    with pytest.raises(D.DuctGPUError) as e:
        gpu_ctx.helm3d(rhs.copy(order="F"), "d", 5.0, np.array([0.0, 1.0]))
    assert e.value.code == D.ESTATE
    gpu_ctx.set_operators("d", ops.ED, ops.PD, ops.PDM1)
    with pytest.raises(D.DuctGPUError) as e:
        gpu_ctx.helm3d(rhs.copy(order="F"), "d", 5.0, np.array([0.0, 1.0]))
    assert e.value.code == D.ESTATE
    gpu_ctx.set_operators("n", ops.EN, ops.PN, ops.PNM1, ops.iofzero)
    sol = gpu_ctx.helm3d(rhs.copy(order="F"), "d", 5.0, np.array([0.0, 1.0]))
    ref, _ = oracle.helm3d(rhs, ops, "d", 5.0, np.array([0.0, 1.0]))
    assert rel(sol, ref) < TOL_KERNEL


@pytest.mark.parametrize("m", [9, 33, 64, 65, 129, 193])
def test_imported_operators_on_grid_only_setup(gpu_ctx, oracle, m):
    nm = 4
    ops = oracle.Ops(m)
    gpu_ctx.pseudomat_ex(m)
    gpu_ctx.set_operators("d", ops.ED, ops.PD, ops.PDM1)
    gpu_ctx.set_operators("n", ops.EN, ops.PN, ops.PNM1, ops.iofzero)
    assert not gpu_ctx.folded("d") and not gpu_ctx.folded("n")
    xalp = np.array([0.0, 0.5, 3.0, 11.0])
    rhs = synth.chebyshev_rhs(m, m, nm, seed=100 + m, ib=0)
    for bound, lam in (("d", 4.0e6), ("d", 0.0), ("n", 0.0)):
        ref, _ = oracle.helm3d(rhs, ops, bound, lam, xalp)
        sol = gpu_ctx.helm3d(rhs.copy(order="F"), bound, lam, xalp)
        assert rel(sol, ref) < TOL_KERNEL, (bound, lam)
        if bound == "n":
            io = ops.iofzero
            assert sol[io, io, 0] == 0.0 or abs(sol[io, io, 0]) < 1e-13 * np.abs(sol[:, :, 0]).max()


@pytest.mark.parametrize("m", [17, 33, 65, 129])
def test_gauge_point_on_own_operators(gpu_ctx, oracle, m):
    """The library's own eigen-decomposition with the reference's iofzero:
    the kx=0 pressure equals the oracle's pointwise (no constant removed)."""
    nm = 3
    ops = oracle.Ops(m)
    gpu_ctx.pseudomat(m)
    gpu_ctx.set_gauge_point(ops.iofzero)
    xalp = np.array([0.0, 0.5, 2.0])
    rhs = synth.chebyshev_rhs(m, m, nm, seed=200 + m, ib=0)
    ref, _ = oracle.helm3d(rhs, ops, "n", 0.0, xalp)
    sol = gpu_ctx.helm3d(rhs.copy(order="F"), "n", 0.0, xalp)
    io = ops.iofzero
    assert abs(sol[io, io, 0]) <= 1e-13 * np.abs(sol[:, :, 0]).max()
    for k in range(nm):
        assert rel(sol[:, :, k], ref[:, :, k]) < TOL_NEU, k
    # the default (0) goes back to the operators' own smallest-|E| position
    gpu_ctx.set_gauge_point(0)
    E, P, Q, io_own = gpu_ctx.get_operators("n", m - 2)
    sol2 = gpu_ctx.helm3d(rhs.copy(order="F"), "n", 0.0, xalp)
    assert abs(sol2[io_own, io_own, 0]) <= 1e-13 * np.abs(sol2[:, :, 0]).max()
    d = sol2[1:-1, 1:-1, 0] - sol[1:-1, 1:-1, 0]
    assert np.max(np.abs(d - d.mean())) < 1e-9 * np.abs(sol[:, :, 0]).max()
    with pytest.raises(D.DuctGPUError) as e:
        gpu_ctx.set_gauge_point(m - 1)
    assert e.value.code == D.EARG
