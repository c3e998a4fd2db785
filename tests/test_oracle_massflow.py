"""The mass-flow restatement (src/operators.F:2205-2344) against known
answers, no GPU: at lambda -> 0 the particular solution is the laminar
profile over -dpval, so its flow rate is -Q/dpval with the classical
series Q; impose_mass_flow hits the target flow exactly."""
import numpy as np

DPVAL_ASPECT1 = 3.39344926982230   # src/operators.F:2498


def laminar_flow():
    i = np.arange(1, 200001, 2, dtype=np.float64)
    return 4.0 / 3.0 * (1.0 - 192.0 / np.pi ** 5 * np.sum(np.tanh(i * np.pi / 2) / i ** 5)) * DPVAL_ASPECT1


def test_poisson_limit_gives_laminar_flow(oracle):
    ops = oracle.Ops(65)
    _, pf = oracle.precomp_mass_flow(ops, 1.0, [1.0e20], 1.0)
    assert abs(pf[0] + laminar_flow() / DPVAL_ASPECT1) < 1e-10


def test_impose_hits_target(oracle):
    ops = oracle.Ops(33)
    pu, pf = oracle.precomp_mass_flow(ops, 2e-4, [8 / 15, 2 / 15, 1 / 3], 1 / 4400, aspect=2.0)
    rng = np.random.default_rng(3)
    u = np.asfortranarray(rng.standard_normal((33, 33, 2)) + 0j)
    for krk in (1, 2, 3):
        v, _, _ = oracle.impose_mass_flow(u, 1.25, krk, pu, pf, 1, aspect=2.0)
        _, flow, _ = oracle.impose_mass_flow(v, 0.0, krk, pu, pf, 0, aspect=2.0)
        assert abs(flow - 1.25) < 1e-12
        assert np.array_equal(v[:, :, 0].imag, u[:, :, 0].imag)
