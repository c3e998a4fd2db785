"""Captured solves (CUDA graphs) and the reference's own GPU entry points
(transpose_gpu_, mat_invdiag_gpu_) through the C-ABI."""
import ctypes as C

import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu


def test_graph_replay_square_substep(gpu_ctx):
    m, nm = 65, 8
    gpu_ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nm)
    fields = []
    for bound, lam, seed in (("d", 4.0e6, 1), ("d", 4.0e6, 2), ("d", 4.0e6, 3), ("n", 0.0, 4)):
        rhs = synth.chebyshev_rhs(m, m, nm, seed=seed, ib=0)
        r, s = gpu_ctx.device_array(rhs.shape), gpu_ctx.device_array(rhs.shape)
        r.upload(rhs)
        fields.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, bound=bound, host=rhs))
    gpu_ctx.solve_fields_dev(fields)
    gpu_ctx.synchronize()
    direct = [f["sol"].download() for f in fields]
    gid = gpu_ctx.graph_create(fields)
    for f in fields:                       # new right-hand sides, same buffers
        f["rhs"].upload(2.0 * f["host"])
    for _ in range(3):
        gpu_ctx.graph_launch(gid)
    gpu_ctx.synchronize()
    for f, d in zip(fields, direct):
        got = f["sol"].download()
        assert np.max(np.abs(got - 2.0 * d)) <= 1e-12 * np.max(np.abs(d))
    gpu_ctx.graph_destroy(gid)
    for f in fields:
        f["rhs"].free()
        f["sol"].free()


def test_graph_replay_cfg1_batch_matches_direct(gpu_ctx):
    """The benchmark's step: u, v, w, p at my = 129 with 64 modes (the
    warp-specialised flip-symmetric passes), two graphs over two buffer sets
    replayed alternately, equal bit for bit to direct calls."""
    m, nm = 129, 64
    gpu_ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nm)
    specs = (("d", 4.0e6), ("d", 4.0e6), ("d", 4.0e6), ("n", 0.0))
    sets, keep = [], []
    try:
        for s in range(2):
            fl = []
            for i, (bound, lam) in enumerate(specs):
                rhs = synth.chebyshev_rhs(m, m, nm, seed=100 * s + i, ib=0)
                r, o = gpu_ctx.device_array(rhs.shape), gpu_ctx.device_array(rhs.shape)
                r.upload(rhs)
                keep += [r, o]
                fl.append(dict(rhs=r, sol=o, xalp=xalp, alambda=lam, ib=0, bound=bound))
            sets.append(fl)
        direct = []
        for fl in sets:
            gpu_ctx.solve_fields_dev(fl)
            gpu_ctx.synchronize()
            direct.append([f["sol"].download() for f in fl])
        gids = [gpu_ctx.graph_create(fl) for fl in sets]
        for fl in sets:
            for f in fl:
                f["sol"].upload(np.zeros((m, m, nm), dtype=np.complex128, order="F"))
        for k in range(4):
            gpu_ctx.graph_launch(gids[k % 2])
        gpu_ctx.synchronize()
        for fl, d in zip(sets, direct):
            for f, ref in zip(fl, d):
                assert np.array_equal(f["sol"].download(), ref)
        for g in gids:
            gpu_ctx.graph_destroy(g)
    finally:
        for x in keep:
            x.free()


def test_graph_replay_rect(gpu_ctx):
    gpu_ctx.pseudomat_temp(0, 33, 65, 1.0, 2.0)
    gpu_ctx.pseudomat_temp(1, 49, 97, 1.0, 2.0, ("n", "n"), ("n", "n"))
    fields = []
    for slot, (my, mz), lam in ((0, (33, 65), 100.0), (1, (49, 97), 0.0)):
        rhs = synth.chebyshev_rhs(my, mz, 4, seed=slot, ib=0)
        r, s = gpu_ctx.device_array(rhs.shape), gpu_ctx.device_array(rhs.shape)
        r.upload(rhs)
        fields.append(dict(rhs=r, sol=s, xalp=np.arange(4.0), alambda=lam, ib=0, slot=slot))
    gpu_ctx.solve_rect_fields_dev(fields)
    gpu_ctx.synchronize()
    direct = [f["sol"].download() for f in fields]
    gid = gpu_ctx.graph_create(fields, rect=True)
    gpu_ctx.graph_launch(gid)
    gpu_ctx.synchronize()
    for f, d in zip(fields, direct):
        assert np.array_equal(f["sol"].download(), d)
    gpu_ctx.graph_destroy(gid)
    for f in fields:
        f["rhs"].free()
        f["sol"].free()


@pytest.mark.parametrize("nx,ny", [(32, 32), (127, 127), (33, 70), (1, 5)])
def test_reference_transpose_and_invdiag(gpu_ctx, nx, ny):
    L = D.lib()
    rng = np.random.default_rng(nx * ny)
    A = np.asfortranarray(rng.standard_normal((nx, ny)))
    ED = np.asfortranarray(rng.standard_normal((nx, ny)) - 5.0)
    dA, dC, dE = (gpu_ctx.device_array(s, np.float64) for s in ((nx, ny), (ny, nx), (nx, ny)))
    dA.upload(A)
    dE.upload(ED)
    h = C.c_size_t(0)
    ix, iy, al = C.c_int(nx), C.c_int(ny), C.c_double(1.0)
    pa, pc, pe = C.c_size_t(dA.ptr), C.c_size_t(dC.ptr), C.c_size_t(dE.ptr)
    assert L.transpose_gpu_(C.byref(h), C.byref(ix), C.byref(iy), C.byref(al), C.byref(pa), C.byref(pc)) == 0
    gpu_ctx.synchronize()
    assert np.array_equal(dC.download(), A.T)
    dF = gpu_ctx.device_array((nx, ny), np.float64)
    dF.upload(A)
    pf, po = C.c_size_t(dF.ptr), C.c_size_t(dA.ptr)
    lam = C.c_double(0.25)
    assert L.mat_invdiag_gpu_(C.byref(h), C.byref(ix), C.byref(iy), C.byref(lam), C.byref(pf), C.byref(pe), C.byref(po)) == 0
    gpu_ctx.synchronize()
    assert np.allclose(dA.download(), A / (ED - 0.25), rtol=1e-15, atol=0)
    for d in (dA, dC, dE, dF):
        d.free()
