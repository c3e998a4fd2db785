"""The Shen-Legendre solver (helm3d_shen path) through the C-ABI against
the oracle, exact polynomial solutions, the batched launch and a captured
graph.

Tolerance: both sides are FP64, but the generalized eigenvectors come from
cuSOLVER's sygvd here and LAPACK's dsygv in the oracle; their round-off
differs by ~eps * cond(P), so results agree to TOL relative to the field
norm, and the exact solutions to TOL_EXACT absolutely."""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

from test_oracle_shen import manufactured

pytestmark = pytest.mark.gpu
TOL = 1e-12
TOL_EXACT = 1e-12


def rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


# my - 1 = 2^a 3^b (the transform's sizes); 163 is the largest below 191
@pytest.mark.parametrize("m", [9, 17, 33, 65, 129, 163])
@pytest.mark.parametrize("bound", ["d", "n"])
def test_against_oracle(gpu_ctx, oracle, m, bound):
    nm = 4
    f = synth.chebyshev_rhs(m, m, nm, seed=m, ib=0)
    xalp = np.array([0.0, 0.5, 1.0, 7.0])
    lam = 0.0 if bound == "n" else 2.5
    ref, ref_after = oracle.helm3d_shen(f, oracle.Shen(m, bound), lam, xalp, ib=0)
    rhs = f.copy(order="F")
    got = gpu_ctx.helm3d_shen(rhs, bound, lam, xalp, ib=0, ipro=0)
    assert rel(got, ref) < TOL
    assert rel(rhs, ref_after) < 1e-14
    assert np.all(got[:, :, 0].imag == 0)


@pytest.mark.parametrize("bound", ["d", "n"])
@pytest.mark.parametrize("lam", [0.5, 4.0e6])
def test_manufactured(gpu_ctx, oracle, bound, lam):
    m = 65
    u, f = manufactured(oracle, m, bound, lam)
    rhs = np.zeros((m, m, 2), dtype=np.complex128, order="F")
    rhs[:, :, 0] = f
    rhs[:, :, 1] = f * (1 - 1j)
    got = gpu_ctx.helm3d_shen(rhs, bound, lam, np.zeros(2), ib=0, ipro=0)
    scale = max(1.0, np.abs(u).max())
    assert np.abs(got[:, :, 0] - u).max() < TOL_EXACT * scale
    assert np.abs(got[:, :, 1] - u * (1 - 1j)).max() < TOL_EXACT * scale * 2


def test_batched_fields_and_graph(gpu_ctx, oracle):
    """u, v, w (Dirichlet) and p (Neumann) of a substep in one batched call
    and as a captured graph equal the per-field oracle solutions."""
    m, nm = 33, 6
    gpu_ctx.preshen(m, "d")
    gpu_ctx.preshen(m, "n")
    xalp = 0.5 * np.arange(1, nm + 1)
    specs = [("d", 4.0e3, 1), ("d", 4.0e3, 2), ("d", 4.0e3, 3), ("n", 0.0, 4)]
    hosts, refs = [], []
    for bound, lam, seed in specs:
        f = synth.chebyshev_rhs(m, m, nm, seed=seed, ib=1)
        hosts.append(f)
        refs.append(oracle.helm3d_shen(f, oracle.Shen(m, bound), lam, xalp, ib=1)[0])
    dev, fields = [], []
    for (bound, lam, _), f in zip(specs, hosts):
        r, s = gpu_ctx.device_array(f.shape), gpu_ctx.device_array(f.shape)
        r.upload(f)
        dev.append((r, s))
        fields.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=1, bound=bound))
    gpu_ctx.solve_shen_fields_dev(fields)
    gpu_ctx.synchronize()
    for (r, s), ref in zip(dev, refs):
        assert rel(s.download(), ref) < TOL
    # graph replay: rhs is transformed in place, so it is reloaded each time
    gid = gpu_ctx.graph_create(fields, shen=True)
    try:
        for _ in range(2):
            for (r, s), f in zip(dev, hosts):
                r.upload(f)
            gpu_ctx.graph_launch(gid)
            gpu_ctx.synchronize()
            for (r, s), ref in zip(dev, refs):
                assert rel(s.download(), ref) < TOL
    finally:
        gpu_ctx.graph_destroy(gid)
    for r, s in dev:
        r.free()
        s.free()


def test_argument_errors(gpu_ctx):
    with pytest.raises(D.DuctGPUError):
        gpu_ctx.preshen(32, "d")          # even
    with pytest.raises(D.DuctGPUError):
        gpu_ctx.preshen(193, "d")         # above the supported size
    with pytest.raises(D.DuctGPUError):
        gpu_ctx.preshen(33, "x")
