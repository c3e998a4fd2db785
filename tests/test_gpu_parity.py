"""Flip-symmetric GEMM passes (DUCTGPU_PASS_PARITY).

With the same condition on both walls the interior operator commutes with
the reflection of the Gauss-Lobatto points, so ductgpu_pseudomat's operators
split into an even and an odd half block, decomposed on their own: every
pass becomes block diagonal (half the flops).  That is another FP64
eigen-decomposition of the same operator, so it is held to the bounds of the
GPU's own operators in test_gpu_solve.py, and for accuracy against the
extended-precision solution of the discrete operator: Dirichlet fields
within 5e-12 of the oracle (at n >= 128 the difference is the oracle's own
error) with error <= 5 x the oracle's own + 1e-13; Neumann fields within
2e-10 (modulo the gauge constant of the singular mode) with error
<= max(5 x the oracle's own, 1e-13 n^1.5) + 1e-12.
Operators imported with ductgpu_set_operators are applied as given: the
variant then runs the full passes, bit for bit the STAGED result.
"""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-12
TOL_D = 5e-12
TOL_KERNEL = 1e-13
TOL_NEU = 2e-10


def rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


def exact_interior(F, B, P, Q, E, lam, io=None, iters=4):
    """Iterative refinement with a long-double residual of the interior
    problem B U + U B^T - lam U = F (FP64 diagonalisation as preconditioner)."""
    Bl = B.astype(np.longdouble)
    Fl = F[1:-1, 1:-1].astype(np.longdouble)
    U = np.zeros_like(Fl)
    den = E[:, None] + E[None, :] - lam
    if io is not None:
        den[io, io] = np.inf
    for _ in range(iters):
        R = (Fl - (Bl @ U + U @ Bl.T - lam * U)).astype(np.float64)
        d = P @ ((Q @ R @ Q.T) / den) @ P.T
        if io is not None:
            d = d - d[io, io] * np.outer(P[:, io], P[:, io]) / P[io, io] ** 2
        U = U + d.astype(np.longdouble)
    return U.astype(np.float64)


@pytest.fixture
def parity(gpu_ctx):
    gpu_ctx.set_pass_kernel(D.PASS_PARITY)
    yield gpu_ctx
    gpu_ctx.set_pass_kernel(-1)   # the library's defaults


@pytest.mark.parametrize("m", [9, 17, 33, 34, 65, 97, 129, 130, 193])
def test_parity_against_oracle(parity, oracle, m):
    ctx = parity
    nm = 3
    ops = oracle.Ops(m)
    ctx.pseudomat(m)
    rhs = synth.chebyshev_rhs(m, m, nm, seed=m, ib=0)
    xalp = np.array([0.0, 1.5, 7.0])
    n = m - 2
    for alam in (4.0e6, 1.0):
        ref_d, _ = oracle.helm3d(rhs, ops, "d", alam, xalp)
        sol_d = ctx.helm3d(rhs.copy(order="F"), "d", alam, xalp, ipro=0)
        # two FP64 decompositions: at n >= 128 their difference is the
        # oracle's own error (up to ~8e-13 against the exact solution)
        assert rel(sol_d, ref_d) < TOL_D
        for k in range(nm):
            for part in (np.real, np.imag):
                if k == 0 and part is np.imag:
                    continue
                X = exact_interior(np.asfortranarray(part(rhs[:, :, k])), ops.D2Bd, ops.PD, ops.PDM1,
                                   ops.ED, alam + xalp[k] ** 2)
                g, o = part(sol_d[1:-1, 1:-1, k]), part(ref_d[1:-1, 1:-1, k])
                assert rel(g, X) <= 5 * rel(o, X) + 1e-13, (alam, k, rel(g, X), rel(o, X))
    ref_n, _ = oracle.helm3d(rhs, ops, "n", 0.0, xalp)
    sol_n = ctx.helm3d(rhs.copy(order="F"), "n", 0.0, xalp)
    for k in range(nm):
        a, b = sol_n[:, :, k], ref_n[:, :, k]
        if k == 0:
            a, b = a - a.mean(), b - b.mean()
        assert rel(a, b) < TOL_NEU, k
    assert np.all(sol_n[:, :, 0].imag == 0)
    for k in range(nm):
        lam = xalp[k] ** 2
        io = ops.iofzero - 1 if lam == 0 else None
        for part in (np.real, np.imag):
            if k == 0 and part is np.imag:
                continue
            X = exact_interior(np.asfortranarray(part(rhs[:, :, k])), ops.D2Bn, ops.PN, ops.PNM1,
                               ops.EN, lam, io)
            g, o = part(sol_n[1:-1, 1:-1, k]), part(ref_n[1:-1, 1:-1, k])
            if io is not None:
                X, g, o = X - X.mean(), g - g.mean(), o - o.mean()
            assert rel(g, X) <= max(5 * rel(o, X), 1e-13 * n ** 1.5) + 1e-12, (k, rel(g, X), rel(o, X))


def test_parity_is_a_different_path(gpu_ctx):
    """The variant really runs the half blocks (its result is not the full
    passes' bit pattern), and agrees with them to rounding."""
    m, nm = 65, 4
    gpu_ctx.pseudomat(m)
    rhs = synth.chebyshev_rhs(m, m, nm, seed=3, ib=0)
    xalp = 0.5 * np.arange(nm)
    try:
        gpu_ctx.set_pass_kernel(D.PASS_STAGED)
        full = gpu_ctx.helm3d(rhs.copy(order="F"), "d", 2.0, xalp)
        gpu_ctx.set_pass_kernel(D.PASS_PARITY)
        half = gpu_ctx.helm3d(rhs.copy(order="F"), "d", 2.0, xalp)
    finally:
        gpu_ctx.set_pass_kernel(-1)
    assert not np.array_equal(full, half)
    assert rel(half, full) < TOL


def test_parity_imported_operators_run_full_passes(parity, oracle):
    ctx = parity
    m, nm = 33, 5
    ops = oracle.Ops(m)
    ctx.pseudomat(m)
    ctx.set_operators("d", ops.ED, ops.PD, ops.PDM1)
    ctx.set_operators("n", ops.EN, ops.PN, ops.PNM1, ops.iofzero)
    rhs = synth.chebyshev_rhs(m, m, nm, seed=5, ib=0)
    xalp = 0.5 * np.arange(nm)
    got = {b: ctx.helm3d(rhs.copy(order="F"), b, lam, xalp) for b, lam in (("d", 3.0), ("n", 0.0))}
    ctx.set_pass_kernel(D.PASS_STAGED)
    for b, lam in (("d", 3.0), ("n", 0.0)):
        full = ctx.helm3d(rhs.copy(order="F"), b, lam, xalp)
        assert np.array_equal(got[b], full)
        ref, _ = oracle.helm3d(rhs, ops, b, lam, xalp)
        assert rel(got[b], ref) < TOL_KERNEL


def test_parity_batched_fields_match_single_solves(parity):
    """One launch sequence over Dirichlet and Neumann fields (singular kx=0
    pressure plane included) equals the fields solved one by one."""
    ctx = parity
    m, nm = 129, 4
    ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nm)
    specs = [("d", 4.0e6), ("d", 1.0), ("n", 0.0)]
    fl, keep, singles = [], [], []
    try:
        for i, (b, lam) in enumerate(specs):
            f = synth.chebyshev_rhs(m, m, nm, seed=20 + i, ib=0)
            singles.append(ctx.helm3d(f.copy(order="F"), b, lam, xalp))
            r, s = ctx.device_array(f.shape), ctx.device_array(f.shape)
            r.upload(f)
            keep += [r, s]
            fl.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, bound=b))
        ctx.solve_fields_dev(fl)
        ctx.synchronize()
        for f, one in zip(fl, singles):
            assert np.array_equal(f["sol"].download(), one)
    finally:
        for x in keep:
            x.free()


def test_warp_specialised_pass_matches_small_batches(parity, oracle):
    """A cfg1-sized batch (4 fields x 64 modes at my = 129: 2048 tiles of 16
    lines, >= 6 per SM) runs the warp-specialised persistent kernel; the same
    fields in batches of 8 modes run the 3-CTA-per-SM kernel.  Same fragment
    order, K order and epilogue arithmetic: equal bit for bit.  A few planes
    are also checked against the oracle (bounds of the module docstring)."""
    ctx = parity
    m, nm, chunk = 129, 64, 8
    ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nm)
    specs = [("d", 4.0e6), ("d", 1.0), ("d", 4.0e6), ("n", 0.0)]
    rhs = [synth.chebyshev_rhs(m, m, nm, seed=60 + i, ib=0) for i in range(len(specs))]
    keep = []
    try:
        big = []
        for (b, lam), f in zip(specs, rhs):
            r, s = ctx.device_array(f.shape), ctx.device_array(f.shape)
            r.upload(f)
            keep += [r, s]
            big.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, bound=b))
        ctx.solve_fields_dev(big)
        ctx.synchronize()
        whole = [f["sol"].download() for f in big]
        for k0 in range(0, nm, chunk):
            small = []
            for (b, lam), f in zip(specs, rhs):
                part = np.asfortranarray(f[:, :, k0:k0 + chunk])
                r, s = ctx.device_array(part.shape), ctx.device_array(part.shape)
                r.upload(part)
                keep += [r, s]
                small.append(dict(rhs=r, sol=s, xalp=xalp[k0:k0 + chunk], alambda=lam, ib=k0, bound=b))
            ctx.solve_fields_dev(small)
            ctx.synchronize()
            for f, w in zip(small, whole):
                assert np.array_equal(f["sol"].download(), w[:, :, k0:k0 + chunk]), k0
        ops = oracle.Ops(m)
        for (b, lam), f, w in zip(specs, rhs, whole):
            for k in (0, 1, 63):
                ref, _ = oracle.helm3d(np.asfortranarray(f[:, :, k:k + 1]), ops, b, lam, xalp[k:k + 1], ib=k)
                got = w[:, :, k:k + 1]
                if b == "n" and k == 0:
                    got, ref = got - got.mean(), ref - ref.mean()
                assert rel(got, ref) < (TOL_D if b == "d" else TOL_NEU), (b, k)
    finally:
        for x in keep:
            x.free()


def test_warp_specialised_pass_hpad32_matches_small_batches(parity):
    """Half blocks of 32 rows (my = 65) in a batch large enough for the
    warp-specialised kernel (4 fields x 128 modes: 2048 tiles) equal the
    same fields in 16-mode batches (the 3-CTA-per-SM kernel) bit for bit."""
    ctx = parity
    m, nm, chunk = 65, 128, 16
    ctx.pseudomat(m)
    xalp = 0.25 * np.arange(nm)
    specs = [("d", 2.0e4), ("d", 3.0), ("n", 0.0), ("n", 1.0)]
    rhs = [synth.chebyshev_rhs(m, m, nm, seed=70 + i, ib=0) for i in range(len(specs))]
    keep = []
    try:
        big = []
        for (b, lam), f in zip(specs, rhs):
            r, s = ctx.device_array(f.shape), ctx.device_array(f.shape)
            r.upload(f)
            keep += [r, s]
            big.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, bound=b))
        ctx.solve_fields_dev(big)
        ctx.synchronize()
        whole = [f["sol"].download() for f in big]
        for k0 in range(0, nm, chunk):
            small = []
            for (b, lam), f in zip(specs, rhs):
                part = np.asfortranarray(f[:, :, k0:k0 + chunk])
                r, s = ctx.device_array(part.shape), ctx.device_array(part.shape)
                r.upload(part)
                keep += [r, s]
                small.append(dict(rhs=r, sol=s, xalp=xalp[k0:k0 + chunk], alambda=lam, ib=k0, bound=b))
            ctx.solve_fields_dev(small)
            ctx.synchronize()
            for f, w in zip(small, whole):
                assert np.array_equal(f["sol"].download(), w[:, :, k0:k0 + chunk]), k0
    finally:
        for x in keep:
            x.free()


def test_adjoint_at_cfg1_size_is_the_transpose(parity):
    """The adjoint of a cfg1-sized batch (warp-specialised kernel on the
    transposed half blocks): <g, S f> = <S^T g, f> for u, v, w and p."""
    ctx = parity
    m, nm = 129, 64
    ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nm)
    specs = [("d", 4.0e6), ("d", 4.0e6), ("d", 4.0e6), ("n", 0.0)]
    keep, fwd, adj, data = [], [], [], []
    try:
        for i, (b, lam) in enumerate(specs):
            f = synth.chebyshev_rhs(m, m, nm, seed=90 + i, ib=0)
            gg = synth.chebyshev_rhs(m, m, nm, seed=95 + i, ib=0)
            a = [ctx.device_array(f.shape) for _ in range(4)]
            a[0].upload(f)
            a[2].upload(gg)
            keep += a
            fwd.append(dict(rhs=a[0], sol=a[1], xalp=xalp, alambda=lam, ib=0, bound=b))
            adj.append(dict(rhs=a[2], sol=a[3], xalp=xalp, alambda=lam, ib=0, bound=b))
            data.append((f, gg, a))
        ctx.solve_fields_dev(fwd)
        ctx.solve_adjoint_fields_dev(adj)
        ctx.synchronize()
        for (b, _), (f, gg, a) in zip(specs, data):
            Sf, STg = a[1].download(), a[3].download()
            lhs = np.vdot(gg.ravel(), Sf.ravel()).real
            rhs_ = np.vdot(STg.ravel(), f.ravel()).real
            scale = np.linalg.norm(gg) * np.linalg.norm(Sf) + np.linalg.norm(STg) * np.linalg.norm(f)
            assert abs(lhs - rhs_) < 1e-13 * scale, (b, lhs, rhs_)
    finally:
        for x in keep:
            x.free()
