"""Pins of the oracle's DNS time step (src/main1.f90:384-723 and the
routines it calls) by known answers:

* fourx (src/fourier.F:1-188): the x transform of a band-limited field is
  exact both ways, and a product formed in physical space keeps only the
  modes 0..mx1 (the 2/3 rule): cos(k x)^2 = 1/2 + cos(2 k x)/2;
* the laminar duct flow (lap U = -dpval, U = 0 on the walls) is a steady
  state of the full RK3/CN step, driven either by the mean pressure
  gradient (icase 1) or by the held flow rate (CMASSFLOW);
* its wall stress integrates the pressure gradient: the four walls of
  wallstressx (src/operators.F:676-710) sum to -dpval area / circumference
  as the grid is refined (algebraically: the corners make the exact
  profile singular);
* a divergence-free perturbation stays divergence-free to rounding through
  the projection step (max_3din, src/operators.F:2524-2550);
* energy_fou / statistics_fou of the laminar field.
"""
import numpy as np
import pytest

from duct_b200 import synth


def test_fourx_round_trip_and_dealiasing(oracle):
    mg, my, nz, M = 24, 3, 2, 8           # mx = 16, mx1 = 7
    rng = np.random.default_rng(0)
    fou = rng.standard_normal((M, my, nz)) + 1j * rng.standard_normal((M, my, nz))
    fou[0] = fou[0].real
    phys = oracle.fourx(fou, mgalx=mg, iopt=1)
    back = oracle.fourx(np.zeros_like(fou), phys, iopt=-1)
    assert np.abs(back - fou).max() < 1e-14
    # cos(3x)^2 = 1/2 + cos(6x)/2; cos(5x)^2 keeps only 1/2 (mode 10 > mx1)
    for k, keep in ((3, True), (5, False)):
        f = np.zeros((M, 1, 1), dtype=complex)
        f[k] = 0.5
        x = oracle.fourx(f, mgalx=mg, iopt=1)
        xn = np.arange(mg) * 2 * np.pi / mg
        assert np.abs(x[:mg, 0, 0] - np.cos(k * xn)).max() < 1e-14
        sq = oracle.fourx(np.zeros_like(f), x * x, iopt=-1)
        ref = np.zeros(M, dtype=complex)
        ref[0] = 0.5
        if keep:
            ref[2 * k] = 0.25
        assert np.abs(sq[:, 0, 0] - ref).max() < 1e-14


def test_derivx(oracle):
    rng = np.random.default_rng(1)
    u = rng.standard_normal((5, 5, 4)) + 1j * rng.standard_normal((5, 5, 4))
    xalp = np.array([0.0, 0.5, 1.0, 1.5])
    d1 = oracle.derivx(u, xalp, 1, scal=2.0)
    d2 = oracle.derivx(u, xalp, 2, scal=3.0)
    assert np.abs(d1 - 2.0 * 1j * xalp * u).max() < 1e-15 * np.abs(d1).max()
    assert np.abs(d2 - (-3.0 * xalp ** 2 * u)).max() < 1e-15 * np.abs(d2).max()


@pytest.mark.parametrize("cmassflow", [True, False])
def test_laminar_flow_is_a_steady_state(oracle, cmassflow):
    m, mg, fnu, dt = 17, 24, 1.0 / 500.0, 1.0e-3
    u, v, w, p, dpval = synth.dns_initial(mg, m, 1.0, 0.0, seed=1)
    d = oracle.Dns(u, v, w, p, mg, 1.0, fnu, dt, cmassflow=cmassflow, dpdx=-fnu * dpval)
    for _ in range(3):
        d.step(stats=True)
    assert np.abs(d.u - u).max() < 1e-13
    assert np.abs(d.v).max() < 1e-15 and np.abs(d.w).max() < 1e-15 and np.abs(d.p).max() < 1e-14
    # wall stress balances the pressure gradient: sum -> -dpval * 4 / 8
    s = np.sum(d.history[-1]["stress4"])
    assert abs(s + dpval / 2.0) < 1e-4 * dpval
    u33, _, _, _, dp33 = synth.dns_initial(mg, 33, 1.0, 0.0, seed=1)
    assert abs(np.sum(oracle.wallstressx(u33)) + dp33 / 2.0) < 2e-6 * dp33
    # energies: no fluctuation; energy2 is the rms of the mean flow
    e = d.history[-1]["energy"]
    assert max(e) < 1e-15
    st = d.statistics()
    assert st["nstat"] == 3
    assert np.abs(st["mean"][0] / 3 - u[:, :, 0].real).max() < 1e-13
    assert np.abs(st["prod"][0] / 3 - u[:, :, 0].real ** 2).max() < 1e-13


def test_divergence_free_through_the_projection(oracle):
    m, mg, fnu, dt = 17, 24, 1.0 / 500.0, 1.0e-3
    u, v, w, p, _ = synth.dns_initial(mg, m, 1.0, 0.1, seed=5)
    xalp = 1.0 * np.arange(u.shape[2])
    assert oracle.max_3din(oracle.div3d(u, v, w, xalp, 1.0)) < 1e-14
    d = oracle.Dns(u, v, w, p, mg, 1.0, fnu, dt, cmassflow=True)
    q0 = d.csum
    for _ in range(2):
        div = d.step()
        assert div < 1e-13
    # the flow rate is held
    _, q1, _ = oracle.impose_mass_flow(d.u, 0.0, 1, d.premassfu, d.premassf, 0)
    assert abs(q1 - q0) < 1e-13 * q0
