"""The CPU oracle against known answers (no GPU).

Pins: the laminar-duct table of the reference's get_dpdx
(src/operators.F:2496-2507: -(dyy+dzz)U = dpval gives max U = 1), the
classical series for the laminar square-duct flow rate, and exact
manufactured polynomial solutions of the discrete Dirichlet and Neumann
problems.
"""
import numpy as np
import pytest

DPVAL_ASPECT1 = 3.39344926982230   # src/operators.F:2498


def laminar(O, m):
    ops = O.Ops(m)
    U = np.full((m, m), -DPVAL_ASPECT1, order="F")
    U[0, :] = U[-1, :] = U[:, 0] = U[:, -1] = 0.0
    return ops, O.solvediag(U, ops, "d", 0.0)


@pytest.mark.parametrize("m", [33, 65])
def test_dpval_gives_unit_max(oracle, m):
    _, U = laminar(oracle, m)
    c = (m - 1) // 2
    assert abs(U.max() - 1.0) < 1e-12
    assert abs(U[c, c] - 1.0) < 1e-12


def test_laminar_mass_flow_series(oracle):
    # Q = (4/3) G [1 - 192/pi^5 sum_{i odd} tanh(i pi/2)/i^5] for [-1,1]^2.
    i = np.arange(1, 200001, 2, dtype=np.float64)
    q = 4.0 / 3.0 * (1.0 - 192.0 / np.pi ** 5 * np.sum(np.tanh(i * np.pi / 2) / i ** 5)) * DPVAL_ASPECT1
    _, U = laminar(oracle, 65)
    mass = oracle.cheb2_integral(oracle.transyz_plane(U, -1))
    assert abs(mass - q) < 1e-10


def _grid(O, m):
    return O.Ops(m).xcol


@pytest.mark.parametrize("m,lam", [(17, 0.0), (33, 4.0e6), (33, 2.5), (49, 100.0)])
def test_manufactured_dirichlet(oracle, m, lam):
    ops = oracle.Ops(m)
    x = ops.xcol
    y, z = np.meshgrid(x, x, indexing="ij")
    u = (1 - y ** 2) * (1 - z ** 2) * (1 + 0.3 * y - 0.2 * z * y)
    # lap u - lam u, exact for a polynomial of degree <= m-1
    def d2(p, v, ax):
        return np.gradient(np.gradient(v, axis=ax), axis=ax)
    # analytic second derivatives of the product
    uyy = (-2 * (1 - z ** 2) * (1 + 0.3 * y - 0.2 * z * y)
           + 2 * (-2 * y) * (1 - z ** 2) * (0.3 - 0.2 * z))
    uzz = (-2 * (1 - y ** 2) * (1 + 0.3 * y - 0.2 * z * y)
           + 2 * (-2 * z) * (1 - y ** 2) * (-0.2 * y))
    f = np.asfortranarray(uyy + uzz - lam * u)
    f[0, :] = f[-1, :] = f[:, 0] = f[:, -1] = 0.0
    U = oracle.solvediag(f, ops, "d", lam)
    assert np.max(np.abs(U - u)) < 1e-11 * max(1.0, np.max(np.abs(u)))


@pytest.mark.parametrize("m,lam", [(17, 3.0), (33, 0.25), (33, 0.0)])
def test_manufactured_neumann(oracle, m, lam):
    ops = oracle.Ops(m)
    x = ops.xcol
    y, z = np.meshgrid(x, x, indexing="ij")
    p = lambda s: s ** 2 * (1 - s ** 2 / 2)          # p'(+-1) = 0
    pp = lambda s: 2 - 6 * s ** 2                     # p''
    u = p(y) * p(z) + 0.5 * p(y)
    f = np.asfortranarray(pp(y) * p(z) + p(y) * pp(z) + 0.5 * pp(y) - lam * u)
    U = oracle.solvediag(f, ops, "n", lam)
    if lam == 0.0:
        # singular mode: the reference pins U(iofzero+1, iofzero+1) = 0
        io = ops.iofzero
        assert abs(U[io, io]) < 1e-12
        U = U - U[io, io] + u[io, io]
    assert np.max(np.abs(U - u)) < 1e-10


def test_transyz_round_trip_and_polynomial(oracle):
    rng = np.random.default_rng(0)
    my, mz, nm = 17, 25, 3
    f = np.asfortranarray(rng.standard_normal((my, mz, nm)) + 1j * rng.standard_normal((my, mz, nm)))
    for d in "yz":
        back = oracle.transyz(oracle.transyz(f, d, -1), d, +1)
        assert np.max(np.abs(back - f)) < 1e-13
    # T_3 along y at the reference's transform nodes x_p = cos(pi p/(my-1))
    xp = np.cos(np.pi * np.arange(my) / (my - 1))
    g = np.zeros((my, mz, 1), dtype=complex, order="F")
    g[:, :, 0] = (4 * xp ** 3 - 3 * xp)[:, None]
    c = oracle.transyz(g, "y", -1)
    expect = np.zeros(my)
    expect[3] = 1.0
    assert np.max(np.abs(c[:, :, 0] - expect[:, None])) < 1e-13


def test_derivyz_polynomial(oracle):
    # coefficients of T_4 in y; derivyz differentiates with respect to the
    # solver's coordinate x = -cos(.) (hence the sign): d/dx T4(-x) = -T4'(-x)
    my, mz = 9, 5
    c = np.zeros((my, mz, 1), dtype=complex, order="F")
    c[4, :, 0] = 1.0 + 2.0j
    d1 = oracle.derivyz(c, "y", 1)
    # T4' = 8 T3 + 8 T1 (d_{k-1} = d_{k+1} + 2k c_k), with the sign flip
    expect = np.zeros(my, dtype=complex)
    expect[3] = -8 * (1 + 2j)
    expect[1] = -8 * (1 + 2j)
    assert np.max(np.abs(d1[:, 0, 0] - expect)) < 1e-12
    d2 = oracle.derivyz(c, "y", 2)
    # T4'' = 48 T2 + 64 T0 ... via the same recurrence twice
    e2 = oracle.derivyz(oracle.derivyz(c, "y", 1), "y", 1)
    assert np.max(np.abs(d2 - e2)) < 1e-12
    dz = oracle.derivyz(np.asfortranarray(np.transpose(c, (1, 0, 2))), "z", 1, aspect=2.0)
    assert np.max(np.abs(dz[0, :, 0] - expect / 2.0)) < 1e-12


def test_pencil_transposes_round_trip(oracle):
    rng = np.random.default_rng(1)
    nm, my, nz = 7, 9, 11
    phys = np.asfortranarray(rng.standard_normal((nm, my, nz)) + 1j * rng.standard_normal((nm, my, nz)))
    p2 = oracle.cxyz2yzx(phys)
    assert p2.shape == (my, nz, nm)
    assert np.array_equal(p2[3, 4, 5], phys[5, 3, 4])
    assert np.array_equal(oracle.cyzx2xyz(p2), phys)


def test_helm3d_matches_planewise_solvediag(oracle):
    from duct_b200 import synth
    m, nm = 17, 4
    f = synth.chebyshev_rhs(m, m, nm, seed=3, ib=0)
    ops = oracle.Ops(m)
    xalp = 0.5 * np.arange(nm)
    sol, rhs_after = oracle.helm3d(f, ops, "d", 10.0, xalp, ib=0)
    assert np.all(rhs_after[0, :, :] == 0) and np.all(rhs_after[:, -1, :] == 0)
    for k in range(nm):
        re = oracle.solvediag(np.asfortranarray(rhs_after[:, :, k].real), ops, "d", 10.0 + xalp[k] ** 2)
        assert np.max(np.abs(sol[:, :, k].real - re)) == 0.0
        if k == 0:
            assert np.all(sol[:, :, k].imag == 0.0)
        else:
            im = oracle.solvediag(np.asfortranarray(rhs_after[:, :, k].imag), ops, "d", 10.0 + xalp[k] ** 2)
            assert np.max(np.abs(sol[:, :, k].imag - im)) == 0.0


# get_dpdx table for aspect ratios 1..4 (src/operators.F:2498-2501)
DPVAL = {1.0: 3.39344926982230, 2.0: 2.19545075660646, 3.0: 2.03778220024811, 4.0: 2.00773897291851}


@pytest.mark.parametrize("aspect,my,mz", [(2.0, 65, 129), (3.0, 49, 145), (4.0, 33, 129), (1.0, 33, 33)])
def test_rectangular_dpval_gives_unit_max(oracle, aspect, my, mz):
    y = oracle.Dir(my, 1.0, "d", "d")
    z = oracle.Dir(mz, aspect, "d", "d")
    f = np.full((my, mz, 1), -DPVAL[aspect] + 0j, order="F")
    f[0, :] = f[-1, :] = f[:, 0] = f[:, -1] = 0.0
    u = oracle.helm3d_temp(f, y, z, 0.0, [0.0])
    assert abs(u.real.max() - 1.0) < 1e-12


def test_rectangular_reduces_to_square(oracle):
    m = 17
    ops = oracle.Ops(m)
    from duct_b200 import synth
    f = synth.chebyshev_rhs(m, m, 2, seed=1)
    f[0, :, :] = f[-1, :, :] = f[:, 0, :] = f[:, -1, :] = 0.0
    xalp = np.array([0.0, 1.0])
    sq, _ = oracle.helm3d(f, ops, "d", 2.0, xalp)
    rc = oracle.helm3d_temp(f, oracle.Dir(m), oracle.Dir(m), 2.0, xalp)
    assert np.max(np.abs(sq - rc)) < 1e-12 * np.max(np.abs(sq))


def test_rectangular_manufactured_mixed_walls(oracle):
    # u = y^3 + z^2 y on [-1,1]x[-2,2]: Dirichlet at y=-1 / z=+2, Neumann at
    # y=+1 / z=-2 with the exact wall values and derivatives
    my, mz, b = 17, 21, 2.0
    y = oracle.Dir(my, 1.0, "d", "n")
    z = oracle.Dir(mz, b, "n", "d")
    yy, zz = np.meshgrid(-np.cos(np.pi * np.arange(my) / (my - 1)),
                         -b * np.cos(np.pi * np.arange(mz) / (mz - 1)), indexing="ij")
    u = yy ** 3 + zz ** 2 * yy
    lam = 0.7
    f = 6 * yy + 2 * yy - lam * u
    bcy = np.zeros((mz, 2, 1), order="F")
    bcy[:, 0, 0] = u[0, :]                              # u(y=-1)
    bcy[:, 1, 0] = 3 * 1.0 + zz[0, :] ** 2              # du/dy(y=+1)
    bcz = np.zeros((my, 2, 1), order="F")
    bcz[:, 0, 0] = 2 * (-b) * yy[:, 0]                  # du/dz(z=-b)
    bcz[:, 1, 0] = u[:, -1]                             # u(z=+b)
    F = np.asfortranarray(f[:, :, None] + 0j)
    sol = oracle.helm3d_temp(F, y, z, lam, [0.0], bcy=bcy, bcz=bcz)
    assert np.max(np.abs(sol[1:-1, 1:-1, 0].real - u[1:-1, 1:-1])) < 1e-10
    assert np.max(np.abs(sol[1:-1, 0, 0].real - u[1:-1, 0])) < 1e-10
    assert np.max(np.abs(sol[-1, 1:-1, 0].real - u[-1, 1:-1])) < 1e-10
