"""Constant mass-flow-rate forcing (precomp_mass_flow / impose_mass_flow,
src/operators.F:2205-2344) through the C-ABI against the oracle."""
import numpy as np
import pytest

from duct_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-12
RK3 = np.array([8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0])   # beta_k of a low-storage RK3


@pytest.mark.parametrize("m", [33, 65])
def test_precomp_matches_oracle(gpu_ctx, oracle, m):
    dt, nu, aspect = 2.0e-4, 1.0 / 4400.0, 1.0
    gpu_ctx.pseudomat(m)
    pu, pf = gpu_ctx.precomp_mass_flow(dt, RK3, nu, aspect)
    rpu, rpf = oracle.precomp_mass_flow(oracle.Ops(m), dt, RK3, nu, aspect)
    assert np.linalg.norm(pu - rpu) / np.linalg.norm(rpu) < TOL
    assert np.max(np.abs(pf - rpf) / np.abs(rpf)) < TOL


def test_impose_reaches_target_flow(gpu_ctx, oracle):
    m, dt, nu, aspect = 65, 2.0e-4, 1.0 / 4400.0, 1.5
    gpu_ctx.pseudomat(m)
    pu, pf = gpu_ctx.precomp_mass_flow(dt, RK3, nu, aspect)
    u = synth.chebyshev_rhs(m, m, 3, seed=7, ib=0)
    # iflag 0: the measured flow rate
    flow = gpu_ctx.impose_mass_flow(u.copy(order="F"), 0.0, 1, 0)
    _, _, ref_flow = oracle.impose_mass_flow(u, 0.0, 1, pu, pf, 0, aspect)
    assert abs(flow - ref_flow) <= TOL * max(1.0, abs(ref_flow))
    # iflag 1 at each RK index: the corrected field has the target flow rate
    target = 1.92783343620839
    for krk in (1, 2, 3):
        got = u.copy(order="F")
        gpu_ctx.impose_mass_flow(got, target, krk, 1)
        ref, _, _ = oracle.impose_mass_flow(u, target, krk, pu, pf, 1, aspect)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < TOL
        assert np.array_equal(got[:, :, 1:], u[:, :, 1:])
        assert abs(gpu_ctx.impose_mass_flow(got, 0.0, 1, 0) - target) < 1e-12
