"""The Chebyshev derivative matrices behind the tensor-core line kernel,
checked on the host (no GPU).  ductgpu_cheb_deriv_matrix builds, in long
double, the matrix of the reference's chain transyz -1 -> derivyz ->
transyz +1 (src/tchebw.f:62-192, src/chebyshev.f90:1-295) along one line;
the kernel applies its flip-symmetric half blocks.  It must equal:

* the oracle's own FP64 chain applied to the unit vectors (each column
  D e_c): relative Frobenius differences measured 3e-16..6e-16 for both
  orders at n = 17..193, held to 5e-15;
* for order 1, minus the reference's closed-form collocation matrix
  cheb_colloc_deriv1 (src/cheb_collocation.F, CHQZ (2.4.31) on x_j =
  cos(pi j / N)): the chain differentiates along the ascending coordinate
  y = -x.  The closed form, even evaluated here in long double, loses
  accuracy with n (the differences x_i - x_j cancel near the walls): max
  differences measured 1.2e-15 (n = 17) .. 1.5e-14 (n = 193) of max |D1|,
  held to 2e-16 n;
* for order 2, the square of the order-1 matrix (long double product):
  measured 4e-17..1.5e-16 of max |D2|, held to 2e-15.
"""
import numpy as np
import pytest

import duct_b200 as D

SIZES = [17, 33, 65, 129, 193]


def chain_matrix(oracle, n, order):
    """The oracle's FP64 chain on the n unit vectors (lines along y)."""
    e = np.zeros((n, n, 1), dtype=np.complex128, order="F")
    for c in range(n):
        e[c, c, 0] = 1.0
    f = oracle.transyz(e, "y", -1)
    d = oracle.derivyz(f, "y", order)
    return oracle.transyz(d, "y", 1)[:, :, 0].real


def chqz_d1(n):
    """cheb_colloc_deriv1 (src/cheb_collocation.F) in long double."""
    N = n - 1
    j = np.arange(n, dtype=np.longdouble)
    x = np.cos(np.longdouble(np.pi) * j / N)
    cbar = np.ones(n, dtype=np.longdouble)
    cbar[0] = cbar[N] = 2
    Dm = np.zeros((n, n), dtype=np.longdouble)
    for i in range(n):
        for k in range(n):
            if i != k:
                Dm[i, k] = (-1) ** (i + k) * cbar[i] / (cbar[k] * (x[i] - x[k]))
    for k in range(1, N):
        Dm[k, k] = -x[k] / (2 * (1 - x[k] ** 2))
    Dm[0, 0] = (2 * N * N + 1) / np.longdouble(6)
    Dm[N, N] = -(2 * N * N + 1) / np.longdouble(6)
    return Dm


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n", SIZES)
def test_matches_the_oracle_chain(oracle, n):
    for order in (1, 2):
        got = D.cheb_deriv_matrix(n, order)
        assert rel(got, chain_matrix(oracle, n, order)) < 5e-15


@pytest.mark.parametrize("n", SIZES)
def test_order1_is_minus_the_collocation_matrix(n):
    got = D.cheb_deriv_matrix(n, 1)
    ref = -chqz_d1(n)
    assert np.abs(got - ref).max() < 2e-16 * n * float(np.abs(ref).max())


@pytest.mark.parametrize("n", SIZES)
def test_order2_is_the_square(n):
    d1 = D.cheb_deriv_matrix(n, 1).astype(np.longdouble)
    d2 = D.cheb_deriv_matrix(n, 2)
    ref = d1 @ d1
    assert np.abs(d2 - ref).max() < 2e-15 * float(np.abs(ref).max())


def test_rejects_bad_sizes():
    for n, order in ((2, 1), (1026, 1), (33, 0), (33, 3)):
        with pytest.raises(D.DuctGPUError):
            D.cheb_deriv_matrix(n, order)
