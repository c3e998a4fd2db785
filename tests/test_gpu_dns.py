"""The DNS time step on the GPU against the oracle (src/main1.f90:384-723
and the routines it calls), through the C-ABI.

* the operators around the solve (laplacian3d, grad3d, div3d, update_uvwp,
  derivx; src/operators.F:278-605, src/fourier.F:120-188) on seeded
  smooth fields, square and rectangular, aspect != 1;
* advection3d with the x-FFT 2/3 de-aliasing and statistics_fou2
  (src/operators.F:9-276, 1957-2004) at mgalx = 16 and 64;
* wallstressx, energy_fou, statistics_fou, max_3din;
* whole RK3/CN steps of the device-resident stepper (graph replay and
  direct launches), with the oracle's LAPACK operators imported (so the
  solves agree to rounding), both flow drivings, and with the GPU's own
  operators.

Tolerances: 1e-12 relative (2-norm) for fields built from one or two
derivative passes on smooth data; the steps at 1e-12 for u, v, w with
imported operators.  The pressure is held to 5e-11: its increment phi
solves the Neumann Poisson problem whose right-hand side div(u*) is a small
difference of large derivative terms, so rounding-level differences of u*
(1e-15) come back amplified by the Neumann operator's conditioning
(measured 3e-12..1.2e-11 after one substep at my = 33, absolute 1e-14);
any two FP64 implementations of the step differ this way.  Statistics at
1e-10 (the bar set for the flow statistics).

The FFT line kernel (set_line_kernel(0)) computes the Chebyshev
coefficients with a half-length DCT-I whose post-step is a scan over the
line; at 129 and 193 points its derivatives differ from the oracle's by
up to 1e-11 (measured on these smooth fields: d/dy 9.4e-12, laplacian
1.7e-11 at 193 x 129), against 3e-13 / 9e-13 for the tensor-core kernel
with operators built in long double.  Its tolerance is 4e-11 from 129
points up.
"""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel())


def smooth(my, mz, nm, seed):
    """Seeded complex (my, mz, nm) field with decaying Chebyshev content and
    a real mode 0 (a velocity-like field)."""
    f = synth.chebyshev_rhs(my, mz, nm, seed=seed, ib=0)
    f[:, :, 0] = f[:, :, 0].real
    return np.asfortranarray(f)


@pytest.fixture(scope="module")
def ctx():
    with D.Context(0) as c:
        yield c


def dev(ctx, a):
    d = ctx.device_array(a.shape)
    d.upload(a)
    return d


@pytest.mark.parametrize("kernel", [1, 2, 0])
@pytest.mark.parametrize("my,mz,aspect", [(33, 33, 1.0), (17, 33, 2.0), (65, 49, 0.5), (193, 129, 1.5),
                                          (145, 257, 2.0)])
def test_line_operators_match_oracle(ctx, oracle, my, mz, aspect, kernel):
    """Every line kernel: the collocation matrices' half blocks on the FP64
    tensor cores (1: 8 lines per CTA, 2: 16) and the FFT chain (0)."""
    ctx.set_line_kernel(kernel)
    tol = 4e-11 if kernel == 0 and max(my, mz) >= 129 else 1e-12
    nm = 6
    xalp = 0.7 * np.arange(nm)
    u, v, w, p = (smooth(my, mz, nm, s) for s in (3, 4, 5, 6))
    du, dv, dw, dp = (dev(ctx, a) for a in (u, v, w, p))
    out = [ctx.device_array(u.shape) for _ in range(3)]
    # laplacian3d, overwrite and accumulate
    ref, _ = oracle.laplacian3d(u, xalp, 0.37, "n", aspect=aspect)
    ctx.laplacian3d_dev(du, out[0], xalp, 0.37, "n", aspect=aspect)
    assert rel(out[0].download(), ref) < tol
    acc = smooth(my, mz, nm, 9)
    out[1].upload(acc)
    ref2, _ = oracle.laplacian3d(u, xalp, -1.5, "+", flap=acc, aspect=aspect)
    ctx.laplacian3d_dev(du, out[1], xalp, -1.5, "+", aspect=aspect)
    assert rel(out[1].download(), ref2) < tol
    # grad3d
    gx, gy, gz = oracle.grad3d(p, xalp, 0.8, "n", aspect=aspect)
    ctx.grad3d_dev(dp, out[0], out[1], out[2], xalp, 0.8, "n", aspect=aspect)
    for o, r in zip(out, (gx, gy, gz)):
        assert rel(o.download(), r) < tol
    # div3d
    ref = oracle.div3d(u, v, w, xalp, 2.5, aspect=aspect)
    ctx.div3d_dev(du, dv, dw, out[0], xalp, 2.5, aspect=aspect)
    assert rel(out[0].download(), ref) < tol
    # derivx
    ref = oracle.derivx(u, xalp, 2, scal=0.3)
    ctx.derivx_dev(du, out[0], xalp, 2, 0.3, "n")
    assert rel(out[0].download(), ref) < 1e-14
    # vorticity, the three components
    for c in (1, 2, 3):
        ref = oracle.vorticity(u, v, w, xalp, c, aspect=aspect)
        ctx.vorticity_dev(du, dv, dw, out[c - 1], xalp, c, aspect=aspect)
        assert rel(out[c - 1].download(), ref) < tol, c
    for a in (du, dv, dw, dp, *out):
        a.free()
    ctx.set_line_kernel(1)


@pytest.mark.parametrize("kernel", [1, 2, 0])
def test_update_uvwp_matches_oracle(ctx, oracle, kernel):
    ctx.set_line_kernel(kernel)
    my, nm, aspect = 33, 5, 1.5
    xalp = 0.5 * np.arange(nm)
    u, v, w, p, phi = (smooth(my, my, nm, s) for s in (11, 12, 13, 14, 15))
    ru, rv, rw, rp, _, _ = oracle.update_uvwp(u, v, w, p, phi, xalp, 29 / 96, 37 / 160, 1e-3, 1 / 2000,
                                              aspect=aspect)
    d = [dev(ctx, a) for a in (u, v, w, p, phi)]
    ctx.update_uvwp_dev(*d, xalp, 29 / 96, 37 / 160, 1e-3, 1 / 2000, aspect=aspect)
    for g, r in zip(d[:4], (ru, rv, rw, rp)):
        assert rel(g.download(), r) < 1e-13
    assert np.array_equal(d[4].download(), phi)     # phi left untouched
    for a in d:
        a.free()
    ctx.set_line_kernel(1)


def test_update_uvwp_rejects_aliased_outputs(ctx):
    """update_uvwp writes p, v and u from one line launch; passing the same
    array as u and v would make two outputs of the launch write one field,
    which the kernels cannot order: the call is refused before any launch."""
    my, nm = 33, 3
    xalp = 0.5 * np.arange(nm)
    d = [dev(ctx, smooth(my, my, nm, s)) for s in (41, 42, 43, 44)]
    before = [a.download() for a in d]
    with pytest.raises(D.DuctGPUError) as e:
        ctx.update_uvwp_dev(d[0], d[0], d[1], d[2], d[3], xalp, 29 / 96, 37 / 160, 1e-3, 1 / 2000)
    assert e.value.code == D.EARG and "writes" in str(e.value)
    for a, b in zip(d, before):
        assert np.array_equal(a.download(), b)
        a.free()


@pytest.mark.parametrize("mgalx,my", [(16, 17), (64, 33), (64, 65)])
def test_advection3d_matches_oracle(ctx, oracle, mgalx, my):
    M = (2 * (mgalx // 3)) // 2
    xalp = 1.0 * np.arange(M)
    u, v, w = (smooth(my, my, M, s) for s in (21, 22, 23))
    a1, a2, a3, st = oracle.advection3d(u, v, w, mgalx, xalp, aspect=1.0, stats=True)
    d = [dev(ctx, a) for a in (u, v, w)]
    out = [ctx.device_array(u.shape) for _ in range(3)]
    work = ctx.device_array((my, my, 5 * M))
    stats2 = ctx.device_array((my, my, 6), np.float64)
    stats2.upload(np.zeros((my, my, 6)))
    ctx.advection3d_dev(*d, *out, work, mgalx, xalp, aspect=1.0, stats2=stats2)
    for o, r in zip(out, (a1, a2, a3)):
        assert rel(o.download(), r) < 1e-12
    assert rel(np.moveaxis(stats2.download(), 2, 0), st) < 1e-13
    for a in (*d, *out, work, stats2):
        a.free()


def test_dealiasing_keeps_modes_below_mx1(ctx, oracle):
    """cos(5x)^2 at mgalx = 16 (modes 0..4): the square's mode 10 is beyond
    the kept modes and must not alias into them."""
    mgalx, my = 16, 17
    M = 5
    xalp = np.arange(M, dtype=float)
    u = np.zeros((my, my, M), dtype=complex, order="F")
    u[:, :, 4] = 0.5              # cos(4x)
    z = np.zeros_like(u)
    a1, a2, a3, st = oracle.advection3d(u, z, z, mgalx, xalp, stats=True)
    d = [dev(ctx, a) for a in (u, z, z)]
    out = [ctx.device_array(u.shape) for _ in range(3)]
    work = ctx.device_array((my, my, 5 * M))
    stats2 = ctx.device_array((my, my, 6), np.float64)
    stats2.upload(np.zeros((my, my, 6)))
    ctx.advection3d_dev(*d, *out, work, mgalx, xalp, stats2=stats2)
    s = np.moveaxis(stats2.download(), 2, 0)
    assert np.abs(s[0] - 0.5).max() < 1e-15          # mean of cos^2
    assert np.abs(out[0].download()).max() < 1e-14    # mode 8 dropped, mode 0 has kx = 0
    assert rel(s, st) < 1e-14
    for a in (*d, *out, work, stats2):
        a.free()


def test_statistics_match_oracle(ctx, oracle):
    my, M = 33, 6
    u, v, w, p = (smooth(my, my, M, s) for s in (31, 32, 33, 34))
    d = [dev(ctx, a) for a in (u, v, w, p)]
    for aspect in (1.0, 2.0):
        assert np.abs(ctx.wallstressx_dev(d[0], aspect) - oracle.wallstressx(u, aspect)).max() < 1e-12 * \
            np.abs(oracle.wallstressx(u, aspect)).max()
        e, e2 = ctx.energy_fou_dev(d[1], aspect)
        re, re2 = oracle.energy_fou(v, aspect)
        assert abs(e - re) < 1e-13 * re and abs(e2 - re2) < 1e-13 * re2
    assert abs(ctx.max_3din_dev(d[2]) - oracle.max_3din(w)) < 1e-15 * oracle.max_3din(w)
    mean = ctx.device_array((my, my, 4), np.float64)
    ppb = ctx.device_array((my, my), np.float64)
    spec = ctx.device_array((M, 7, 4), np.float64)
    for a in (mean, ppb, spec):
        a.upload(np.zeros(a.shape))
    ctx.statistics_fou_dev(*d, mean, ppb, spec)
    ctx.statistics_fou_dev(*d, mean, ppb, spec)
    rm, rp, rs = (np.zeros((my, my, 4), order="F"), np.zeros((my, my), order="F"), np.zeros((M, 7, 4), order="F"))
    L = oracle._dlib()
    for _ in range(2):
        L.orc_statistics_fou(*[oracle._p(oracle._cf(f)) for f in (u, v, w, p)], my, my, M, oracle._p(rm),
                             oracle._p(rp), oracle._p(rs))
    assert rel(mean.download(), rm) < 1e-15
    assert rel(ppb.download(), rp) < 1e-14
    assert rel(spec.download(), rs) < 1e-14
    for a in (*d, mean, ppb, spec):
        a.free()


def _dns_pair(oracle, ctx, m, mgalx, amp, seed, cmassflow, imported, fnu=1.0 / 2000.0, dt=1.0e-3, alp=1.0,
              precision=D.PREC_FP64):
    u, v, w, p, dpval = synth.dns_initial(mgalx, m, alp, amp, seed=seed)
    dpdx = -fnu * dpval
    orc = oracle.Dns(u, v, w, p, mgalx, alp, fnu, dt, cmassflow=cmassflow, dpdx=dpdx)
    if imported:
        ops = oracle.Ops(m)
        ctx.pseudomat_ex(m, D.SETUP_NO_EIGEN)
        ctx.set_operators("d", ops.ED, ops.PD, ops.PDM1)
        ctx.set_operators("n", ops.EN, ops.PN, ops.PNM1, ops.iofzero)
    else:
        ctx.pseudomat(m, m)
    gpu = D.Dns(ctx, mgalx, alp, fnu, dt, cmassflow=cmassflow, dpdx=dpdx, precision=precision)
    gpu.set_fields(u, v, w, p)
    return orc, gpu


@pytest.mark.parametrize("cmassflow", [True, False])
def test_dns_steps_match_oracle(oracle, cmassflow):
    m, mgalx = 33, 64
    with D.Context(0) as ctx:
        orc, gpu = _dns_pair(oracle, ctx, m, mgalx, 0.1, 7, cmassflow, imported=True)
        with gpu:
            for step in range(3):
                orc.step(stats=True)
                gpu.steps(1, stats_every=1)
                got = gpu.fields()
                for g, r in zip(got[:3], (orc.u, orc.v, orc.w)):
                    assert rel(g, r) < 1e-12, step
                assert rel(got[3], orc.p) < 5e-11, step
                for g in got:
                    assert np.all(g[:, :, 0].imag == 0)     # mode 0 stays real
            st, ref = gpu.statistics(), orc.statistics()
            assert st["nstat"] == ref["nstat"] == 3
            for key in ("mean", "prod", "ppb", "spec"):
                assert rel(st[key], ref[key]) < 1e-10, key
            hist = np.array([h["stress4"] + h["energy"] + h["energy2"] for h in orc.history])
            assert st["hist"].shape == hist.shape
            assert np.abs(st["hist"] - hist).max() < 1e-10 * np.abs(hist).max()
            assert st["divmax"][2] == pytest.approx(orc.divmax, rel=1e-6, abs=1e-13)
            assert st["divmax"].max() < 1e-11
            # the first substep's time-step and slip checks (determine_step,
            # slip_velocity_3d) on the physical velocities of the last step
            cf = gpu.cfl()
            dt = 1.0e-3
            assert cf["cfl"] == pytest.approx(dt * orc.history[-1]["remx"], rel=1e-12)
            assert cf["cfl_max"] == pytest.approx(dt * max(h["remx"] for h in orc.history), rel=1e-12)
            assert abs(cf["slip"] - orc.history[-1]["slip"]) < 1e-12
            assert gpu.cfl()["cfl_max"] == 0.0      # reset by the read, no step since
            # the vorticity diagnostics of the recorded steps
            om, oref = gpu.statistics_omg(), orc.statistics_omg()
            assert rel(om["om2"], oref["om2"]) < 1e-10
            assert om["hist"].shape == oref["hist"].shape == (3, 16)
            assert np.abs(om["hist"] - oref["hist"]).max() < 1e-10 * np.abs(oref["hist"]).max()
            assert np.all(oref["hist"][:, 10:] > 0)
            # the reference's ENER log lines of the three recorded steps
            lines = gpu.ener_lines()
            assert len(lines) == 3 and all(len(ln.split()) == 39 for ln in lines)
            ref13 = [D.fortran_e15_8(x) for x in oref["hist"][2, 0:4]]
            assert lines[2].split()[13:17] == [r.strip() for r in ref13] or \
                np.allclose([float(x) for x in lines[2].split()[13:17]], oref["hist"][2, 0:4], rtol=1e-7)


def test_dns_graph_replay_equals_direct_launches(oracle):
    """Substeps replayed as CUDA graphs give bit-identical fields to the
    same substeps launched directly."""
    m, mgalx = 33, 64
    res = []
    for graphs in (True, False):
        with D.Context(0) as ctx:
            _, gpu = _dns_pair(oracle, ctx, m, mgalx, 0.1, 3, True, imported=True)
            with gpu:
                gpu.set_graphs(graphs)
                gpu.steps(3, stats_every=1)
                res.append(gpu.fields() + [gpu.statistics()["prod"]])
    for a, b in zip(*res):
        assert np.array_equal(a, b)


def test_dns_cfg3_size_own_operators(oracle):
    """cfg3's grid (my = 65, mgalx = 64, 21 modes, 5 % perturbation) with
    the GPU's own eigen-decompositions: the step agrees with the oracle to
    the FP64 noise of the Neumann solve, and the flow stays
    divergence-free."""
    fnu = 1.92783343620839 / (4.0 * 2000.0)
    with D.Context(0) as ctx:
        orc, gpu = _dns_pair(oracle, ctx, 65, 64, 0.05, 1, True, imported=False, fnu=fnu, dt=1e-3)
        with gpu:
            orc.step()
            gpu.steps(1)
            got = gpu.fields()
            for g, r in zip(got[:3], (orc.u, orc.v, orc.w)):
                assert rel(g, r) < 1e-11
            assert rel(got[3], orc.p) < 1e-9
            assert gpu.statistics()["divmax"].max() < 1e-10
