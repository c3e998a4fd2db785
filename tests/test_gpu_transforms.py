"""Chebyshev transforms (transyz), derivatives (derivyz) and pencil
transposes through the C-ABI against the oracle.  Tolerances: transforms and
derivatives 1e-13 relative to the largest input magnitude (FFT vs the
oracle's direct sums, both FP64); transposes bit-exact."""
import ctypes as C

import numpy as np
import pytest

import duct_b200 as D

pytestmark = pytest.mark.gpu


def field(my, mz, nm, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((my, mz, nm)) + 1j * rng.standard_normal((my, mz, nm)))


# line lengths 9..193 cover the register-FFT plans (2(n-1) = 16 ... 384);
# 19 (2(n-1) = 36) has no plan and runs the radix-stage kernel
SHAPES = [(9, 17, 2), (33, 33, 3), (129, 65, 2), (193, 49, 2), (145, 33, 1), (65, 193, 1), (19, 13, 2)]


@pytest.mark.parametrize("my,mz,nm", SHAPES)
@pytest.mark.parametrize("cdir", ["y", "z"])
def test_transyz_matches_oracle(gpu_ctx, oracle, my, mz, nm, cdir):
    f = field(my, mz, nm, my + mz)
    for iopt in (-1, 1):
        ref = oracle.transyz(f, cdir, iopt)
        got = gpu_ctx.transyz(f, cdir, iopt)
        assert np.max(np.abs(got - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref))), iopt
    back = gpu_ctx.transyz(gpu_ctx.transyz(f, cdir, -1), cdir, +1)
    assert np.max(np.abs(back - f)) < 1e-13 * np.max(np.abs(f))


@pytest.mark.parametrize("my,mz,nm", SHAPES[:4])
@pytest.mark.parametrize("cdir", ["y", "z"])
@pytest.mark.parametrize("ider", [1, 2])
def test_derivyz_matches_oracle(gpu_ctx, oracle, my, mz, nm, cdir, ider):
    u = field(my, mz, nm, 7)
    # smooth spectrum so the derivative stays O(1)
    k = np.arange(my)[:, None, None] + np.arange(mz)[None, :, None]
    u = np.asfortranarray(u / (1.0 + k) ** 4)
    ref = oracle.derivyz(u, cdir, ider, scal=0.7, aspect=2.0)
    got = gpu_ctx.derivyz(u, cdir, ider, scal=0.7, aspect=2.0)
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
    base = field(my, mz, nm, 8)
    ref2 = oracle.derivyz(u, cdir, ider, scal=-1.5, what="a", du=base, aspect=3.0)
    got2 = gpu_ctx.derivyz(u, cdir, ider, scal=-1.5, what="a", du=base, aspect=3.0)
    assert np.max(np.abs(got2 - ref2)) <= 1e-13 * np.max(np.abs(ref2))


def _dev(ctx, a):
    d = ctx.device_array(a.shape)
    d.upload(a)
    return d


def test_pencil_transposes_bit_exact(gpu_ctx, oracle):
    L = D.lib()
    nm, my, nz = 21, 65, 33
    phys = field(nm, my, nz, 3)
    p_d = _dev(gpu_ctx, phys)
    q_d = gpu_ctx.device_array((my, nz, nm))
    gpu_ctx._check(L.ductgpu_cxyz2yzx_dev(gpu_ctx.h, C.c_void_p(p_d.ptr), C.c_void_p(q_d.ptr), nm, my, nz))
    assert np.array_equal(q_d.download(), oracle.cxyz2yzx(phys))
    r_d = gpu_ctx.device_array((nm, my, nz))
    gpu_ctx._check(L.ductgpu_cyzx2xyz_dev(gpu_ctx.h, C.c_void_p(r_d.ptr), C.c_void_p(q_d.ptr), nm, my, nz))
    assert np.array_equal(r_d.download(), phys)
    for d in (p_d, q_d, r_d):
        d.free()


@pytest.mark.parametrize("nm,my,nz", [(85, 193, 193), (1, 3, 5), (33, 7, 9), (8, 2, 2), (64, 129, 129), (5, 40, 3)])
def test_pencil_transposes_bit_exact_sizes(gpu_ctx, oracle, nm, my, nz):
    """The transposes at the config-4 field and at ragged sizes (tiles of 32
    cut by the array's edges on both sides; tensor-map boxes beyond them)."""
    L = D.lib()
    phys = field(nm, my, nz, nm + my)
    p_d = _dev(gpu_ctx, phys)
    q_d = gpu_ctx.device_array((my, nz, nm))
    gpu_ctx._check(L.ductgpu_cxyz2yzx_dev(gpu_ctx.h, C.c_void_p(p_d.ptr), C.c_void_p(q_d.ptr), nm, my, nz))
    assert np.array_equal(q_d.download(), oracle.cxyz2yzx(phys))
    r_d = gpu_ctx.device_array((nm, my, nz))
    gpu_ctx._check(L.ductgpu_cyzx2xyz_dev(gpu_ctx.h, C.c_void_p(r_d.ptr), C.c_void_p(q_d.ptr), nm, my, nz))
    assert np.array_equal(r_d.download(), phys)
    gpu_ctx.synchronize()
    for d in (p_d, q_d, r_d):
        d.free()


def test_chx2z_chz2x_round_trip(gpu_ctx, oracle):
    L = D.lib()
    my, mz, nm = 33, 33, 17
    u = field(my, mz, nm, 4)
    xy = _dev(gpu_ctx, u)
    xz = gpu_ctx.device_array(u.shape)
    gpu_ctx._check(L.ductgpu_chx2z_dev(gpu_ctx.h, C.c_void_p(xy.ptr), C.c_void_p(xz.ptr), my, mz, nm))
    # xz keeps the (y,z,x) copy, xy holds the x-fastest transpose
    assert np.array_equal(xz.download(), u)
    t = xy.download().ravel(order="F").reshape((nm, my, mz), order="F")
    assert np.array_equal(t, oracle.cyzx2xyz(u))
    gpu_ctx._check(L.ductgpu_chz2x_dev(gpu_ctx.h, C.c_void_p(xy.ptr), C.c_void_p(xz.ptr), my, mz, nm))
    assert np.array_equal(xy.download(), u)
    xy.free()
    xz.free()


def test_transform_argument_errors(gpu_ctx):
    f = field(12, 9, 1, 0)          # 12 - 1 = 11 is not 2^a 3^b
    with pytest.raises(D.DuctGPUError) as e:
        gpu_ctx.transyz(f, "y", -1)
    assert e.value.code == D.EARG
    with pytest.raises(D.DuctGPUError):
        gpu_ctx.transyz(field(9, 9, 1, 0), "x", -1)
    with pytest.raises(D.DuctGPUError):
        gpu_ctx.derivyz(field(9, 9, 1, 0), "y", 3)
