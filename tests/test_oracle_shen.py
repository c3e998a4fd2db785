"""The Shen-Legendre oracle (helm3d_shen -> int2d3d -> solveshen,
src/helm_shen.f90, src/solveshen.f90, src/preshen.f90, src/legendre.f90)
against known answers, no GPU.

Pins: exact polynomial solutions of -lap(u) + lambda u = f (the Galerkin
solution is exact when u lies in the Shen space, degree <= my-1 with the
wall condition), the even/odd decoupling the reference's parity split
relies on, the Legendre-Chebyshev matrices (A B = I, Legendre polynomial
values), and the intended pin of the singular Neumann constant mode.
"""
import numpy as np
import pytest


def _poly(bound):
    if bound == "d":
        P = lambda t: (1 - t ** 2) * (1 + 0.3 * t)
        Pyy = lambda t: -2 * (1 + 0.3 * t) + 2 * (-2 * t) * 0.3
        Q = lambda t: (1 - t ** 2) * (1 - 0.2 * t)
        Qzz = lambda t: -2 * (1 - 0.2 * t) + 2 * (-2 * t) * (-0.2)
    else:   # p'(+-1) = 0: t^2 - t^4/2 and 3t - t^3
        P = lambda t: t ** 2 - t ** 4 / 2 + 0.3 * (3 * t - t ** 3)
        Pyy = lambda t: 2 - 6 * t ** 2 + 0.3 * (-6 * t)
        Q = lambda t: t ** 2 - t ** 4 / 2 - 0.2 * (3 * t - t ** 3)
        Qzz = lambda t: 2 - 6 * t ** 2 - 0.2 * (-6 * t)
    return P, Pyy, Q, Qzz


def manufactured(O, m, bound, lam):
    """u on the collocation nodes and f = -lap(u) + lam u."""
    x = O.Ops(m).xcol
    y, z = np.meshgrid(x, x, indexing="ij")
    P, Pyy, Q, Qzz = _poly(bound)
    u = P(y) * Q(z)
    f = -(Pyy(y) * Q(z) + P(y) * Qzz(z)) + lam * u
    return u, f


@pytest.mark.parametrize("m", [17, 33, 65])
@pytest.mark.parametrize("bound", ["d", "n"])
@pytest.mark.parametrize("lam", [0.5, 100.0])
def test_manufactured(oracle, m, bound, lam):
    u, f = manufactured(oracle, m, bound, lam)
    rhs = np.zeros((m, m, 2), dtype=np.complex128, order="F")
    rhs[:, :, 0] = f
    rhs[:, :, 1] = f * (1 + 2j)
    sol, after = oracle.helm3d_shen(rhs, oracle.Shen(m, bound), lam, np.zeros(2), ib=0)
    assert np.abs(sol[:, :, 0] - u).max() < 1e-13
    assert np.abs(sol[:, :, 1] - u * (1 + 2j)).max() < 1e-13
    assert np.all(sol[:, :, 0].imag == 0)
    # rhs comes back as its Chebyshev coefficients (transyz y, z; iopt -1)
    c = oracle.transyz(oracle.transyz(rhs, "y", -1), "z", -1)
    assert np.abs(after - c).max() < 1e-13 * np.abs(c).max()


@pytest.mark.parametrize("m", [17, 65, 129])
@pytest.mark.parametrize("bound", ["d", "n"])
def test_parity_split_is_exact(oracle, m, bound):
    """The reference keeps only the even/odd blocks of P, P^-1 S^-1 and A
    (src/preshen.f90:203-287); the full operators differ from that by
    round-off only."""
    assert oracle.Shen(m, bound).parity_leak() < 1e-13


@pytest.mark.parametrize("m", [9, 33])
def test_legendre_chebyshev_matrices(oracle, m):
    s = oracle.Shen(m, "d")
    assert np.abs(s.A @ s.B - np.eye(m)).max() < 1e-12
    # column k of B holds the Chebyshev coefficients of L_k
    t = np.linspace(-1, 1, 7)
    T = np.cos(np.outer(np.arccos(t), np.arange(m)))
    for k in range(m):
        Lk = np.polynomial.legendre.legval(t, np.eye(m)[k])
        assert np.abs(T @ s.B[:, k] - Lk).max() < 1e-12


def test_neumann_constant_mode_pin(oracle):
    """At lambda = 0 the Neumann problem is singular; the reference's solV
    pins the constant Shen coefficient (src/solveshen.f90:424-432): the
    result differs from the exact solution by a constant only."""
    m = 33
    u, f = manufactured(oracle, m, "n", 0.0)
    rhs = np.zeros((m, m, 1), dtype=np.complex128, order="F")
    rhs[:, :, 0] = f
    sol, _ = oracle.helm3d_shen(rhs, oracle.Shen(m, "n"), 0.0, np.zeros(1), ib=0)
    d = sol[:, :, 0].real - u
    assert np.abs(d - d.mean()).max() < 1e-12
