"""Adjoint (reverse-mode) gradient through one RK3/CN step, config 3:
square duct, mgalx = 64 (21 modes), my = mz = 65, Lx = 2 pi, Re_b = 2000,
laminar profile plus a 5 % seeded divergence-free perturbation, CMASSFLOW.
J = the wall stress of u summed over the four walls (wallstressx,
src/operators.F:676-710) after one step, differentiated with respect to a
seeded body force f of amplitude 1e-3 (h += (akk+bkk) f in every substep,
as the reference's forcings enter, src/main1.f90 (vi-b)).

* the forced step itself matches the oracle's forced step;
* the adjoint gradient's directional derivatives <dJ/df, e> match central
  finite differences (h = 1e-6) of J on the GPU and of J on the reference
  path (the oracle's step), for seeded directions e;
* the gradient vanishes where the forward map ignores f (wall points,
  the imaginary part of mode 0).

Tolerances.  J is a wall-normal derivative: evaluating it amplifies the
rounding of u by the weights' size, ~N^2 eps, so J itself carries ~1e-12
relative noise (measured: GPU and oracle J differ by 1.1e-12).  Central
differences with the config's h = 1e-6 therefore see 1e-12 |J| / 2h ~ 1e-6
of noise on directional derivatives of order 1e-3: agreement to 1e-3
relative is asked there.  With h = 1e-3 that noise is ~1e-9, and the
central difference's own error is O(h^2) times the third derivative of a J
that is nearly linear in f (f enters the advection products only from the
second substep on): agreement to 1e-6 relative.
"""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu

Q_LAMINAR = 1.9081638750


def cfg3():
    c = synth.dns_config("cfg3")
    c["fnu"] = Q_LAMINAR / (4.0 * c["re_b"])
    return c


def seeded_field(m, M, seed, amp):
    rng = np.random.default_rng(seed)
    f = np.zeros((m, m, M), dtype=np.complex128, order="F")
    k = min(M, 6)
    f[:, :, :k] = rng.standard_normal((m, m, k)) + 1j * rng.standard_normal((m, m, k))
    f[:, :, 0] = f[:, :, 0].real
    return np.asfortranarray(amp * f / np.abs(f).max())


def dot(a, b):
    return float(np.sum(np.real(np.conj(a) * b)))


@pytest.fixture(scope="module")
def case(oracle):
    c = cfg3()
    m, mg, alp = c["my"], c["mgalx"], c["alp"]
    M = (2 * (mg // 3)) // 2
    u, v, w, p, _ = synth.dns_initial(mg, m, alp, c["amp"], seed=3)
    f = [seeded_field(m, M, 100 + i, 1e-3) for i in range(3)]
    return dict(c=c, m=m, mg=mg, alp=alp, M=M, state=(u, v, w, p), f=f)


@pytest.fixture(scope="module")
def gpu(case):
    c = case["c"]
    with D.Context(0) as ctx:
        ctx.pseudomat(case["m"])
        with D.Dns(ctx, case["mg"], case["alp"], c["fnu"], c["dt"], cmassflow=True) as d:
            d.set_fields(*case["state"])
            d.set_forcing(case["f"])
            d.set_graphs(False)
            yield ctx, d


def test_forced_step_matches_oracle(oracle, case):
    c = case["c"]
    m = case["m"]
    orc = oracle.Dns(*case["state"], case["mg"], case["alp"], c["fnu"], c["dt"], cmassflow=True)
    orc.set_forcing(case["f"])
    orc.step()
    ops = oracle.Ops(m)
    with D.Context(0) as ctx:
        ctx.pseudomat_ex(m, D.SETUP_NO_EIGEN)
        ctx.set_operators("d", ops.ED, ops.PD, ops.PDM1)
        ctx.set_operators("n", ops.EN, ops.PN, ops.PNM1, ops.iofzero)
        with D.Dns(ctx, case["mg"], case["alp"], c["fnu"], c["dt"], cmassflow=True) as d:
            d.set_fields(*case["state"])
            d.set_forcing(case["f"])
            J = d.wallstress_after(1)
            d.steps(1)
            got = d.fields()
    for g, r in zip(got[:3], (orc.u, orc.v, orc.w)):
        assert np.linalg.norm(g - r) < 1e-12 * np.linalg.norm(r)
    # J: wall-normal derivatives at the walls summed with weights of order
    # N^2 (the oracle through its DCT, the GPU with the equivalent
    # physical-space weights), so two roundings differ by ~N^2 eps |J|
    Jr = float(np.sum(oracle.wallstressx(orc.u)))
    assert abs(J - Jr) < 1e-11 * abs(Jr)


def test_gradient_matches_finite_differences(gpu, case):
    ctx, d = gpu
    f = case["f"]
    J0, g = d.grad_wallstress()
    assert J0 == pytest.approx(d.wallstress_after(1), rel=1e-14)
    # the forward map ignores f at the walls (the Dirichlet solve zeroes the
    # rhs walls) and the imaginary part of mode 0
    for gc in g:
        assert np.all(gc[0, :, :] == 0) and np.all(gc[-1, :, :] == 0)
        assert np.all(gc[:, 0, :] == 0) and np.all(gc[:, -1, :] == 0)
        assert np.all(gc[:, :, 0].imag == 0)
    assert np.abs(g).max() > 0
    for h, tol in ((1e-6, 1e-3), (1e-3, 1e-6)):
        for seed in (7, 8, 9):
            e = [seeded_field(case["m"], case["M"], seed * 10 + i, 1.0) for i in range(3)]
            d.set_forcing([fc + h * ec for fc, ec in zip(f, e)])
            jp = d.wallstress_after(1)
            d.set_forcing([fc - h * ec for fc, ec in zip(f, e)])
            jm = d.wallstress_after(1)
            fd = (jp - jm) / (2 * h)
            ad = sum(dot(gc, ec) for gc, ec in zip(g, e))
            assert abs(fd - ad) < tol * abs(ad), (h, seed, fd, ad)
    d.set_forcing(f)


def test_gradient_matches_reference_path(oracle, gpu, case):
    """<dJ/df, e> against central differences of the oracle's forced step
    (the reference's CPU path)."""
    ctx, d = gpu
    c = case["c"]
    _, g = d.grad_wallstress()
    for h, tol in ((1e-6, 1e-3), (1e-3, 1e-6)):
        for seed in (11, 12):
            e = [seeded_field(case["m"], case["M"], seed * 10 + i, 1.0) for i in range(3)]
            js = []
            for s in (1.0, -1.0):
                orc = oracle.Dns(*case["state"], case["mg"], case["alp"], c["fnu"], c["dt"], cmassflow=True)
                orc.set_forcing([fc + s * h * ec for fc, ec in zip(case["f"], e)])
                orc.step()
                js.append(float(np.sum(oracle.wallstressx(orc.u))))
            fd = (js[0] - js[1]) / (2 * h)
            ad = sum(dot(gc, ec) for gc, ec in zip(g, e))
            assert abs(fd - ad) < tol * abs(ad), (h, seed, fd, ad)
