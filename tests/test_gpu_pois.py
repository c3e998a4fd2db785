"""The Galerkin-basis Neumann solver (pseudopois / solvepois) through the
C-ABI: exact polynomial solutions, the kx=0 gauge, parity with the oracle on
the same (imported LAPACK) operators, and the batched complex form.

At lambda = 0 the reference pins the grid point (iofzero+1, iofzero+1),
where iofzero is the position of the zero eigenvalue in LAPACK's eigenvalue
order; cuSOLVER orders differently, so with its own operators the GPU
solution agrees with the oracle's up to a constant (the null vector is the
constant), and exactly once the oracle's operators are imported."""
import ctypes as C

import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

from test_oracle_pois import manufactured

pytestmark = pytest.mark.gpu
TOL = 1e-12


def gpu_iofzero(ctx, m):
    io = C.c_int()
    assert D.lib().ductgpu_get_operators(ctx.h, b"p", None, None, None, C.byref(io)) == D.OK
    return io.value


@pytest.mark.parametrize("m", [17, 33, 65, 129])
@pytest.mark.parametrize("lam", [1.5, 400.0])
def test_manufactured(gpu_ctx, oracle, m, lam):
    gpu_ctx.pseudopois(m)
    u, f = manufactured(oracle, m, lam)
    g = gpu_ctx.solvepois(np.asfortranarray(f), lam)
    assert np.abs(g - u).max() < 1e-11 * np.abs(u).max()


@pytest.mark.parametrize("m", [33, 129, 193])
def test_singular_mode_up_to_constant(gpu_ctx, oracle, m):
    gpu_ctx.pseudopois(m)
    u, f = manufactured(oracle, m, 0.0)
    g = gpu_ctx.solvepois(np.asfortranarray(f), 0.0)
    io = gpu_iofzero(gpu_ctx, m)
    assert abs(g[io, io]) < 1e-13 * np.abs(g).max()        # this solver's own pin
    d = g - u
    assert np.abs(d - d[io, io]).max() < 5e-11 * np.abs(u).max()


@pytest.mark.parametrize("m", [33, 129])
@pytest.mark.parametrize("lam", [0.0, 2.0])
def test_matches_oracle_on_imported_operators(gpu_ctx, oracle, m, lam):
    p = oracle.Pois(m)
    gpu_ctx.pseudopois(m)
    gpu_ctx.set_operators("p", p.EN, p.PN, p.PNM1, p.iofzero)
    rng = np.random.default_rng(m)
    f = np.asfortranarray(rng.standard_normal((m, m)))
    g = gpu_ctx.solvepois(f, lam)
    r = oracle.solvepois(f, p, lam)
    assert np.linalg.norm(g - r) / np.linalg.norm(r) < TOL


def test_batched_complex_fields(gpu_ctx, oracle):
    m, nm = 65, 4
    p = oracle.Pois(m)
    gpu_ctx.pseudopois(m)
    gpu_ctx.set_operators("p", p.EN, p.PN, p.PNM1, p.iofzero)
    xalp = np.array([0.0, 1.0, 2.0, 3.0])
    hosts = [synth.chebyshev_rhs(m, m, nm, seed=s, ib=0) for s in (3, 4)]
    dev, fields = [], []
    for f in hosts:
        r, s = gpu_ctx.device_array(f.shape), gpu_ctx.device_array(f.shape)
        r.upload(f)
        dev.append((r, s))
        fields.append(dict(rhs=r, sol=s, xalp=xalp, alambda=0.0, ib=0, bound="n"))
    gpu_ctx.solve_pois_fields_dev(fields)
    gpu_ctx.synchronize()
    for (r, s), f in zip(dev, hosts):
        got = s.download()
        assert np.all(got[:, :, 0].imag == 0)
        for k in range(nm):
            lam = xalp[k] ** 2
            ref = oracle.solvepois(np.asfortranarray(f[:, :, k].real), p, lam)
            assert np.linalg.norm(got[:, :, k].real - ref) / np.linalg.norm(ref) < TOL
            if k:
                refi = oracle.solvepois(np.asfortranarray(f[:, :, k].imag), p, lam)
                assert np.linalg.norm(got[:, :, k].imag - refi) / np.linalg.norm(refi) < TOL
        r.free()
        s.free()
