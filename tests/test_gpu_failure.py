"""Failure detection on the GPU without a fault: a bounded device-side wait
that runs out is reported to the host as a status, and the context stays
usable afterwards.

ductgpu_selftest_wait_timeout launches one CTA whose wait -- the bounded
mbarrier wait of the pipelined pass kernels -- is on a barrier that nothing
completes (a flag that nothing sets); after its poll limit it raises the
context's error word instead of spinning on.
"""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth


@pytest.mark.gpu
def test_wait_that_runs_out_reports_timeout_and_context_stays_usable(gpu_ctx, oracle):
    L = D.lib()
    h = gpu_ctx.h
    gpu_ctx.synchronize()                                        # nothing pending
    assert L.ductgpu_selftest_wait_timeout(h, 4096) == D.OK      # the launch itself succeeds
    assert L.ductgpu_synchronize(h) == D.ETIMEOUT                # the wait ran out
    assert "bounded device-side wait" in gpu_ctx.last_error()
    assert L.ductgpu_synchronize(h) == D.OK                      # read once, then cleared

    # the same context still solves correctly
    m, nm = 17, 3
    gpu_ctx.pseudomat(m)
    ops = oracle.Ops(m)
    xalp = 0.5 * np.arange(nm)
    rhs = synth.chebyshev_rhs(m, m, nm, seed=5, ib=0)
    ref, _ = oracle.helm3d(rhs, ops, "d", 3.0, xalp)
    sol = gpu_ctx.helm3d(rhs.copy(order="F"), "d", 3.0, xalp)
    assert np.max(np.abs(sol - ref)) <= 1e-11 * np.max(np.abs(ref))
