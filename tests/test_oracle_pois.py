"""The Galerkin-basis Neumann solver (pseudopois / solvepois,
src/pseudopois.f90, src/solvepois.f90) against known answers, no GPU.

In the basis phi_j = T_j - j^2/(j+2)^2 T_{j+2} (phi_j'(+-1) = 0) the
collocated operator B2 B^-1 is the exact second derivative of every
polynomial of degree <= my-1 with zero end slopes, so such a solution is
reproduced exactly, walls and corners (evaluated from the basis) included;
at lambda = 0 the result is pinned to U(iofzero+1, iofzero+1) = 0 and
differs from the exact one by a constant."""
import numpy as np
import pytest


def poly(t, a):
    """t^2 - t^4/2 + a (3t - t^3) and its second derivative: zero slope at +-1."""
    return t ** 2 - t ** 4 / 2 + a * (3 * t - t ** 3), 2 - 6 * t ** 2 + a * (-6 * t)


def manufactured(O, m, lam):
    x = O.Ops(m).xcol
    y, z = np.meshgrid(x, x, indexing="ij")
    P, Pyy = poly(y, 0.3)
    Q, Qzz = poly(z, -0.2)
    u = P * Q
    f = Pyy * Q + P * Qzz - lam * u
    return u, f


@pytest.mark.parametrize("m", [17, 33, 65])
@pytest.mark.parametrize("lam", [1.5, 400.0])
def test_manufactured(oracle, m, lam):
    u, f = manufactured(oracle, m, lam)
    U = oracle.solvepois(np.asfortranarray(f), oracle.Pois(m), lam)
    assert np.abs(U - u).max() < 1e-11 * np.abs(u).max()


def test_singular_mode_pinned(oracle):
    m = 33
    u, f = manufactured(oracle, m, 0.0)
    p = oracle.Pois(m)
    U = oracle.solvepois(np.asfortranarray(f), p, 0.0)
    io = p.iofzero
    assert abs(U[io, io]) < 1e-13
    d = U - u
    assert np.abs(d - d[io, io]).max() < 1e-10


def test_null_vector_is_constant(oracle):
    p = oracle.Pois(17)
    v = p.PN[:, p.iofzero - 1]
    assert abs(p.EN[p.iofzero - 1]) < 1e-9
    assert np.abs(v / v[0] - 1.0).max() < 1e-9
