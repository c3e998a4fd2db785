"""The adjoint (transposed-eigenbasis) solve through the C-ABI.

Checks: (1) against the transpose of the oracle's dense helm3d matrix
(the FP64 transpose of the reference path, built column by column from unit
right-hand sides) with the oracle's LAPACK operators imported; (2) the
dot-product identity <g, S f> = <S^T g, f> for batched u, v, w, p fields at
65 x 65 with both gauges; (3) the gradient of a wall-shear functional of the
solution with respect to a body forcing against central finite differences
(h = 1e-6)."""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-12


def dense_helm3d(oracle, ops, bound, lam):
    """Real (m^2 x m^2) matrix of the oracle's helm3d map of one mode != 0."""
    m = ops.m
    N = m * m
    E = np.zeros((m, m, N), dtype=np.complex128, order="F")
    for k in range(N):
        E[k % m, k // m, k] = 1.0
    sol, _ = oracle.helm3d(E, ops, bound, lam, np.zeros(N), ib=1)
    return sol.real.reshape(N, N, order="F")


def imported(ctx, oracle, m):
    ops = oracle.Ops(m)
    ctx.pseudomat(m)
    ctx.set_operators("d", ops.ED, ops.PD, ops.PDM1)
    ctx.set_operators("n", ops.EN, ops.PN, ops.PNM1, ops.iofzero)
    return ops


@pytest.mark.parametrize("bound,lam", [("d", 2.5), ("d", 4.0e6), ("n", 3.0), ("n", 0.0)])
def test_matches_oracle_transpose(gpu_ctx, oracle, bound, lam):
    m = 11
    ops = imported(gpu_ctx, oracle, m)
    S = dense_helm3d(oracle, ops, bound, lam)
    rng = np.random.default_rng(17)
    g = np.asfortranarray(rng.standard_normal((m, m, 3)) + 1j * rng.standard_normal((m, m, 3)))
    got = gpu_ctx.helm3d_adjoint(g, bound, lam, np.zeros(3), ib=1)
    N = m * m
    ref = np.empty_like(g)
    for k in range(3):
        gr = g[:, :, k].reshape(N, order="F")
        ref[:, :, k] = (S.T @ gr.real + 1j * (S.T @ gr.imag)).reshape(m, m, order="F")
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < TOL
    # mode 0: real output, real part as above
    got0 = gpu_ctx.helm3d_adjoint(g[:, :, :1], bound, lam, np.zeros(1), ib=0)
    assert np.all(got0.imag == 0)
    assert np.linalg.norm(got0.real - ref[:, :, :1].real) / np.linalg.norm(ref[:, :, :1].real) < TOL


def inner(a, b):
    return float(np.sum(a.real * b.real + a.imag * b.imag))


@pytest.mark.parametrize("gauge", [D.GAUGE_POINT, D.GAUGE_MEAN])
def test_dot_product_identity_batched(gpu_ctx, gauge):
    m, nm = 65, 6
    gpu_ctx.pseudomat(m)
    gpu_ctx.set_gauge(gauge)
    try:
        xalp = 0.5 * np.arange(nm)
        specs = [("d", 4.0e3), ("d", 4.0e3), ("d", 4.0e3), ("n", 0.0)]
        fs = [synth.chebyshev_rhs(m, m, nm, seed=40 + i, ib=0) for i in range(4)]
        gs = [synth.chebyshev_rhs(m, m, nm, seed=80 + i, ib=0) for i in range(4)]
        arrs, fwd, adj = [], [], []
        for (bound, lam), f, g in zip(specs, fs, gs):
            a = [gpu_ctx.device_array(f.shape) for _ in range(4)]
            a[0].upload(f)
            a[2].upload(g)
            arrs.append(a)
            fwd.append(dict(rhs=a[0], sol=a[1], xalp=xalp, alambda=lam, ib=0, bound=bound))
            adj.append(dict(rhs=a[2], sol=a[3], xalp=xalp, alambda=lam, ib=0, bound=bound))
        gpu_ctx.solve_fields_dev(fwd)
        gpu_ctx.solve_adjoint_fields_dev(adj)
        gpu_ctx.synchronize()
        for (bound, _), a, f, g in zip(specs, arrs, fs, gs):
            Sf, STg = a[1].download(), a[3].download()
            lhs, rhs = inner(g, Sf), inner(STg, f)
            scale = np.linalg.norm(g) * np.linalg.norm(Sf) + np.linalg.norm(STg) * np.linalg.norm(f)
            assert abs(lhs - rhs) < 1e-13 * scale, (bound, lhs, rhs)
            assert np.array_equal(a[2].download(), g)        # the cotangent input is read only
            for x in a:
                x.free()
    finally:
        gpu_ctx.set_gauge(D.GAUGE_POINT)


def test_wall_shear_gradient_matches_finite_differences(gpu_ctx):
    """J(f) = sum over the four walls of the Clenshaw-Curtis integral of the
    wall-normal derivative of u = S f (mode 0, Dirichlet, the implicit
    viscous step); dJ/df = S^T c with c = dJ/du."""
    m, lam = 33, 2.0 / (1.0 / 2000.0 * 1.0e-3)
    gpu_ctx.pseudomat(m)
    x = -np.cos(np.pi * np.arange(m) / (m - 1))
    # first-derivative matrix on the nodes (CHQZ), for the functional only
    c_ = np.ones(m)
    c_[0] = c_[-1] = 2.0
    Dm = np.zeros((m, m))
    for i in range(m):
        for j in range(m):
            if i != j:
                Dm[i, j] = c_[i] / c_[j] * (-1.0) ** (i + j) / (x[i] - x[j])
        Dm[i, i] = -Dm[i].sum()          # rows of D annihilate constants
    w = np.zeros(m)
    N = m - 1
    for j in range(m):
        s = sum((1.0 if 2 * k == N else 2.0) * np.cos(2 * np.pi * k * j / N) / (4 * k * k - 1)
                for k in range(1, N // 2 + 1))
        w[j] = (1.0 if j in (0, N) else 2.0) / N * (1.0 - s)
    c = np.zeros((m, m))
    c += np.outer(-Dm[0, :], w)       # -du/dy at y = -1, integrated over z
    c += np.outer(Dm[-1, :], w)       # +du/dy at y = +1
    c += np.outer(w, -Dm[0, :])       # -du/dz at z = -1
    c += np.outer(w, Dm[-1, :])       # +du/dz at z = +1
    rng = np.random.default_rng(5)
    f0 = 1.0e-3 * rng.standard_normal((m, m))

    def J(f):
        rhs = np.asfortranarray(f.reshape(m, m, 1) + 0j)
        u = gpu_ctx.helm3d(rhs, "d", lam, [0.0], ib=0)
        return float(np.sum(c * u[:, :, 0].real))

    grad = gpu_ctx.helm3d_adjoint(np.asfortranarray(c.reshape(m, m, 1) + 0j), "d", lam, [0.0], ib=0)[:, :, 0].real
    h = 1.0e-6
    for _ in range(3):
        e = rng.standard_normal((m, m))
        fd = (J(f0 + h * e) - J(f0 - h * e)) / (2 * h)
        ad = float(np.sum(grad * e))
        assert abs(fd - ad) <= 1e-7 * abs(ad)
