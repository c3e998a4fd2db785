"""Rectangular / general-wall solve (helm3d_temp path) through the C-ABI
against the oracle, the reference's laminar-duct table, and the batched
multi-duct launch.  Tolerances as in test_gpu_solve: 1e-12 for problems
without a Neumann pair, 2e-10 (FP64 eigen-decomposition noise) otherwise."""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu
DPVAL = {1.0: 3.39344926982230, 2.0: 2.19545075660646, 3.0: 2.03778220024811, 4.0: 2.00773897291851}
# the four ducts of the uneven batch: (my, mz), aspect, modes
DUCTS = [((65, 65), 1.0, 32), ((65, 129), 2.0, 48), ((49, 145), 3.0, 64), ((33, 129), 4.0, 96)]


def rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


@pytest.mark.parametrize("shape,aspect,nm", DUCTS)
def test_laminar_table(gpu_ctx, shape, aspect, nm):
    my, mz = shape
    f = np.full((my, mz, 1), -DPVAL[aspect] + 0j, order="F")
    f[0, :] = f[-1, :] = f[:, 0] = f[:, -1] = 0.0
    u = gpu_ctx.helm3d_temp(f, 0.0, [0.0], a=1.0, b=aspect, ipro=0)
    assert abs(u.real.max() - 1.0) < 1e-12


@pytest.mark.parametrize("by,bz", [(("d", "d"), ("d", "d")), (("d", "n"), ("n", "d")),
                                   (("n", "d"), ("d", "n")), (("n", "n"), ("n", "n"))])
def test_against_oracle_with_walls(gpu_ctx, oracle, by, bz):
    my, mz, b, nm = 33, 49, 1.5, 3
    rng = np.random.default_rng(5)
    f = synth.chebyshev_rhs(my, mz, nm, seed=9, ib=0)
    bcy = np.asfortranarray(rng.standard_normal((mz, 2, nm)))
    bcz = np.asfortranarray(rng.standard_normal((my, 2, nm)))
    xalp = np.array([0.0, 1.0, 4.0])
    lam = 3.0
    y, z = oracle.Dir(my, 1.0, *by), oracle.Dir(mz, b, *bz)
    ref = oracle.helm3d_temp(f, y, z, lam, xalp, bcy=bcy, bcz=bcz)
    got = gpu_ctx.helm3d_temp(f.copy(order="F"), lam, xalp, a=1.0, b=b, bcy=bcy, bcz=bcz, by=by, bz=bz, ipro=0)
    tol = 1e-12 if "n" not in by + bz else 2e-10
    assert rel(got, ref) < tol
    assert np.all(got[:, :, 0].imag == 0)


def test_all_neumann_singular_gauge(gpu_ctx, oracle):
    my, mz, b = 33, 65, 2.0
    f = synth.chebyshev_rhs(my, mz, 2, seed=4, ib=0)
    xalp = np.array([0.0, 0.5])
    y, z = oracle.Dir(my, 1.0, "n", "n"), oracle.Dir(mz, b, "n", "n")
    ref = oracle.helm3d_temp(f, y, z, 0.0, xalp)
    got = gpu_ctx.helm3d_temp(f.copy(order="F"), 0.0, xalp, b=b, by=("n", "n"), bz=("n", "n"), ipro=0)
    a, r = got[:, :, 0] - got[:, :, 0].mean(), ref[:, :, 0] - ref[:, :, 0].mean()
    assert rel(a, r) < 2e-10
    assert rel(got[:, :, 1], ref[:, :, 1]) < 2e-10
    gpu_ctx.set_gauge(D.GAUGE_MEAN)
    try:
        gm = gpu_ctx.helm3d_temp(f.copy(order="F"), 0.0, xalp, b=b, by=("n", "n"), bz=("n", "n"))
    finally:
        gpu_ctx.set_gauge(D.GAUGE_POINT)
    wy = oracle.transyz_plane  # noqa: F841  (integral check below via cheb2_integral)
    c = oracle.transyz_plane(np.asfortranarray(gm[:, :, 0].real), -1)
    assert abs(oracle.cheb2_integral(c, aspect=b)) < 1e-11 * np.abs(gm).max()


UNEVEN = {}


@pytest.mark.parametrize("fold,launches", [(0, 4), (1, 12), (2, 1)])
def test_uneven_batch(gpu_ctx, oracle, fold, launches):
    """The four ducts x (3 Dirichlet velocities + Neumann pressure) -- 16
    fields -- in one batched call equal the per-duct oracle solutions: on
    the full operators one launch per GEMM pass (fold 0); on the
    flip-symmetric half blocks (fold 1, the default) the fields grouped by
    their half-block sizes (y: all 32 rows; z: 32, 64 and 96 rows for mz =
    65, 129, 145: three groups), each group's four passes on a stream of its
    own, 12 launches; or the whole solve as one persistent launch (fold 2),
    bit-identical to the grouped launches (the same tile code and K
    order)."""
    gpu_ctx.set_rect_fold(fold)
    nu, dt = 1.0 / 4400.0, 5.0e-4
    h = 2.0 / (nu * dt)
    fields, refs = [], []
    for slot, ((my, mz), aspect, nm) in enumerate(DUCTS):
        gpu_ctx.pseudomat_temp(slot, my, mz, 1.0, aspect)          # Dirichlet walls
        gpu_ctx.pseudomat_temp(4 + slot, my, mz, 1.0, aspect, ("n", "n"), ("n", "n"))
        xalp = 1.0 * np.arange(nm)
        yd, zd = oracle.Dir(my, 1.0), oracle.Dir(mz, aspect)
        yn, zn = oracle.Dir(my, 1.0, "n", "n"), oracle.Dir(mz, aspect, "n", "n")
        for fld in range(4):
            neu = fld == 3
            f = synth.chebyshev_rhs(my, mz, nm, seed=10 * slot + fld, ib=0)
            lam = 0.0 if neu else h
            ref = oracle.helm3d_temp(f, yn if neu else yd, zn if neu else zd, lam, xalp)
            r, s = gpu_ctx.device_array(f.shape), gpu_ctx.device_array(f.shape)
            r.upload(f)
            fields.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, slot=(4 + slot) if neu else slot))
            refs.append((ref, neu))
    gpu_ctx.profile(True)
    gpu_ctx.profile_reset()
    gpu_ctx.solve_rect_fields_dev(fields)
    gpu_ctx.synchronize()
    ms, npass = gpu_ctx.profile_read(D.K_PASS_FP64)
    gpu_ctx.profile(False)
    gpu_ctx.set_rect_fold(1)
    assert npass == launches
    sols = [f["sol"].download() for f in fields]
    UNEVEN[fold] = [a.copy() for a in sols]    # the checks below shift the pressure fields
    if fold == 1:
        # replayed from a captured graph (the groups' streams become parallel
        # branches of it): bit-identical to the direct call
        gpu_ctx.set_rect_fold(1)
        gid = gpu_ctx.graph_create(fields, rect=True)
        for f in fields:
            f["sol"].upload(np.zeros(f["sol"].shape, dtype=complex, order="F"))
        for _ in range(2):
            gpu_ctx.graph_launch(gid)
        gpu_ctx.synchronize()
        gpu_ctx.graph_destroy(gid)
        for f, a in zip(fields, UNEVEN[1]):
            assert np.array_equal(f["sol"].download(), a)
    if fold == 2 and 1 in UNEVEN:
        for a, b in zip(sols, UNEVEN[1]):
            assert np.array_equal(a, b)
    for f, (ref, neu), got in zip(fields, refs, sols):
        if neu:
            got[:, :, 0] -= got[:, :, 0].mean()
            ref = ref.copy()
            ref[:, :, 0] -= ref[:, :, 0].mean()
            assert rel(got, ref) < 2e-10
        else:
            assert rel(got, ref) < 1e-12
        f["rhs"].free()
        f["sol"].free()
