"""ctypes view of the CPU oracle (test infrastructure only).

Used by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
bench.py as the checker.  Arrays use the reference's shapes in Fortran order:
a complex field is ``(my, mz, nmodes)`` complex128, a real plane ``(my, mz)``.
"""
import ctypes as C
import os

import numpy as np

from . import build_oracle

_lib = None


class _Ops(C.Structure):
    _fields_ = [("m", C.c_int)] + [(n, C.POINTER(C.c_double)) for n in (
        "xcol", "DC", "D2", "ED", "EDim", "PD", "PDM1", "EN", "ENim", "PN", "PNM1")] + [
        ("iofzero", C.c_int), ("wanted", C.c_double), ("AM1", C.c_double * 16),
        ("D2Bd", C.POINTER(C.c_double)), ("D2Bn", C.POINTER(C.c_double))]


class _Dir(C.Structure):
    _fields_ = [("m", C.c_int), ("s", C.c_double), ("b1", C.c_char), ("b2", C.c_char)] + [
        (n, C.POINTER(C.c_double)) for n in ("D", "D2", "E", "P", "PM1", "B")]


class _Pois(C.Structure):
    _fields_ = [("m", C.c_int)] + [(n, C.POINTER(C.c_double)) for n in ("EN", "PN", "PNM1", "PNT")] + [
        ("iofzero", C.c_int), ("wanted", C.c_double)]


class _Shen(C.Structure):
    _fields_ = [("m", C.c_int), ("bound", C.c_char)] + [
        (n, C.POINTER(C.c_double)) for n in ("b", "M", "S", "E", "P", "PSM1", "A", "B")]


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        L = C.CDLL(path)
        P = C.c_void_p
        L.orc_pseudomat.argtypes = [C.c_int, C.POINTER(_Ops)]
        L.orc_ops_free.argtypes = [C.POINTER(_Ops)]
        L.orc_solvediag.argtypes = [P, C.POINTER(_Ops), C.c_char, C.c_double]
        L.orc_helm3d.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_char,
                                 C.c_double, C.POINTER(_Ops), C.c_int]
        L.orc_tcheb.argtypes = [P, C.c_long, C.c_long, C.c_long, C.c_int, C.c_int]
        L.orc_transyz.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_char, C.c_int]
        L.orc_transyz_plane.argtypes = [P, C.c_int, C.c_int, C.c_int]
        L.orc_derivyz.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_char, C.c_int,
                                  C.c_double, C.c_char, C.c_double]
        L.orc_cheb2_integral.argtypes = [P, C.c_int, C.c_int, C.c_double]
        L.orc_cheb2_integral.restype = C.c_double
        L.orc_cxyz2yzx.argtypes = [P, P, C.c_int, C.c_int, C.c_int]
        L.orc_cyzx2xyz.argtypes = [P, P, C.c_int, C.c_int, C.c_int]
        L.orc_set_blas_threads.argtypes = [C.c_int]
        L.orc_pseudomat_temp.argtypes = [C.c_int, C.c_double, C.c_char, C.c_char, C.POINTER(_Dir)]
        L.orc_dir_free.argtypes = [C.POINTER(_Dir)]
        L.orc_solvediag_temp.argtypes = [P, C.POINTER(_Dir), C.POINTER(_Dir), C.c_double, P, P, C.c_int]
        L.orc_helm3d_temp.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_double,
                                      C.POINTER(_Dir), C.POINTER(_Dir), P, P, C.c_int]
        L.orc_shen_setup.argtypes = [C.c_int, C.c_char, C.POINTER(_Shen)]
        L.orc_shen_free.argtypes = [C.POINTER(_Shen)]
        L.orc_shen_parity_leak.argtypes = [C.POINTER(_Shen)]
        L.orc_shen_parity_leak.restype = C.c_double
        L.orc_solveshen.argtypes = [P, C.POINTER(_Shen), C.c_double]
        L.orc_helm3d_shen.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_double,
                                      C.POINTER(_Shen), C.c_int]
        L.orc_precomp_mass_flow.argtypes = [C.POINTER(_Ops), C.c_double, P, C.c_int, C.c_double,
                                            C.c_double, P, P]
        L.orc_impose_mass_flow.argtypes = [P, C.c_int, P, C.c_int, C.c_int, C.c_double, P, P, C.c_int]
        L.orc_impose_mass_flow.restype = C.c_double
        L.orc_pseudopois.argtypes = [C.c_int, C.POINTER(_Pois)]
        L.orc_pois_free.argtypes = [C.POINTER(_Pois)]
        L.orc_solvepois.argtypes = [P, C.POINTER(_Pois), C.c_double]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags.f_contiguous or a.ndim <= 1
    return a.ctypes.data_as(C.c_void_p)


class Ops:
    """Result of pseudomat('d',m) + pseudomat('n',m) (src/pseudomat.f90)."""

    def __init__(self, m):
        self._s = _Ops()
        info = lib().orc_pseudomat(m, C.byref(self._s))
        if info != 0:
            raise RuntimeError("orc_pseudomat failed, info=%d" % info)
        self.m = m
        n = m - 2
        s = self._s

        def v(ptr, *shape):
            return np.ctypeslib.as_array(ptr, shape=(int(np.prod(shape)),)).reshape(
                shape, order="F").copy(order="F")
        self.xcol = v(s.xcol, m)
        self.DC = v(s.DC, m, m)
        self.D2 = v(s.D2, m, m)
        self.ED, self.EDim = v(s.ED, n), v(s.EDim, n)
        self.PD, self.PDM1 = v(s.PD, n, n), v(s.PDM1, n, n)
        self.EN, self.ENim = v(s.EN, n), v(s.ENim, n)
        self.PN, self.PNM1 = v(s.PN, n, n), v(s.PNM1, n, n)
        self.D2Bd, self.D2Bn = v(s.D2Bd, n, n), v(s.D2Bn, n, n)
        self.iofzero = s.iofzero
        self.wanted = s.wanted
        self.AM1 = np.array(list(s.AM1)).reshape((4, 4), order="F")

    def __del__(self):
        try:
            lib().orc_ops_free(C.byref(self._s))
        except Exception:
            pass


class Dir:
    """One direction of pseudomaty_temp / pseudomatz_temp
    (src/pseudomat_temp.f90): points m, half-width s, BCs b1 (at -s), b2."""

    def __init__(self, m, s=1.0, b1="d", b2="d"):
        self._s = _Dir()
        info = lib().orc_pseudomat_temp(int(m), float(s), b1.encode(), b2.encode(), C.byref(self._s))
        if info != 0:
            raise RuntimeError("orc_pseudomat_temp failed, info=%d" % info)
        self.m, self.s, self.b1, self.b2 = m, s, b1, b2
        n = m - 2

        def v(ptr, *shape):
            return np.ctypeslib.as_array(ptr, shape=(int(np.prod(shape)),)).reshape(
                shape, order="F").copy(order="F")
        self.D, self.D2 = v(self._s.D, m, m), v(self._s.D2, m, m)
        self.E, self.P, self.PM1, self.B = v(self._s.E, n), v(self._s.P, n, n), v(self._s.PM1, n, n), v(self._s.B, n, n)

    def __del__(self):
        try:
            lib().orc_dir_free(C.byref(self._s))
        except Exception:
            pass


def precomp_mass_flow(ops, dtp, alphak, fnu, aspect=1.0):
    """precomp_mass_flow (src/operators.F:2205-2289): returns (premassfu
    (m,m,mrk), premassf (mrk,))."""
    alphak = np.ascontiguousarray(alphak, dtype=np.float64)
    m, mrk = ops.m, alphak.shape[0]
    pu = np.zeros((m, m, mrk), order="F")
    pf = np.zeros(mrk)
    rc = lib().orc_precomp_mass_flow(C.byref(ops._s), float(dtp), _p(alphak), mrk, float(fnu),
                                     float(aspect), _p(pu), _p(pf))
    if rc:
        raise RuntimeError("orc_precomp_mass_flow: %d" % rc)
    return pu, pf


def impose_mass_flow(u, csum, krk, premassfu, premassf, iflag, aspect=1.0):
    """impose_mass_flow (src/operators.F:2291-2344) on a complex (my,mz,...)
    field; returns (u_after, csum_after, sumg)."""
    u = np.array(u, dtype=np.complex128, order="F")
    my, mz = u.shape[:2]
    cs = C.c_double(float(csum))
    pu = np.asfortranarray(premassfu, dtype=np.float64)
    pf = np.ascontiguousarray(premassf, dtype=np.float64)
    sumg = lib().orc_impose_mass_flow(C.byref(cs), int(krk), _p(u), my, mz, float(aspect), _p(pu), _p(pf),
                                      int(iflag))
    return u, cs.value, sumg


class Pois:
    """pseudopois(m): the Galerkin-basis Neumann operators (src/pseudopois.f90)."""

    def __init__(self, m):
        self._s = _Pois()
        info = lib().orc_pseudopois(int(m), C.byref(self._s))
        if info != 0:
            raise RuntimeError("orc_pseudopois failed, info=%d" % info)
        self.m = m
        n = m - 2

        def v(ptr, *shape):
            return np.ctypeslib.as_array(ptr, shape=(int(np.prod(shape)),)).reshape(
                shape, order="F").copy(order="F")
        self.EN, self.PN, self.PNM1, self.PNT = v(self._s.EN, n), v(self._s.PN, n, n), v(self._s.PNM1, n, n), \
            v(self._s.PNT, n, n)
        self.iofzero = self._s.iofzero

    def __del__(self):
        try:
            lib().orc_pois_free(C.byref(self._s))
        except Exception:
            pass


def solvepois(U, pois, xlambda):
    """solvepois on a real (m,m) plane (interior = rhs); returns the solution."""
    U = np.array(U, dtype=np.float64, order="F")
    lib().orc_solvepois(_p(U), C.byref(pois._s), float(xlambda))
    return U


class Shen:
    """preshen(bound) + leg_cheb_mat for m (odd) points (src/preshen.f90)."""

    def __init__(self, m, bound):
        self._s = _Shen()
        info = lib().orc_shen_setup(int(m), bound.encode(), C.byref(self._s))
        if info != 0:
            raise RuntimeError("orc_shen_setup failed, info=%d" % info)
        self.m, self.bound = m, bound
        n = m - 2

        def v(ptr, *shape):
            return np.ctypeslib.as_array(ptr, shape=(int(np.prod(shape)),)).reshape(
                shape, order="F").copy(order="F")
        self.b = v(self._s.b, m)
        self.M, self.S = v(self._s.M, n, n), v(self._s.S, n, n)
        self.E, self.P, self.PSM1 = v(self._s.E, n), v(self._s.P, n, n), v(self._s.PSM1, n, n)
        self.A, self.B = v(self._s.A, m, m), v(self._s.B, m, m)

    def parity_leak(self):
        return lib().orc_shen_parity_leak(C.byref(self._s))

    def __del__(self):
        try:
            lib().orc_shen_free(C.byref(self._s))
        except Exception:
            pass


def solveshen(U, shen, xlambda):
    """solveshen on one real (m,m) plane of Chebyshev coefficients."""
    U = np.array(U, dtype=np.float64, order="F")
    lib().orc_solveshen(_p(U), C.byref(shen._s), float(xlambda))
    return U


def helm3d_shen(rhs, shen, alambda, xalp, ib=0, nthreads=1):
    """helm3d_shen on a complex (my,mz,nmodes) field: returns (sol, rhs_after)
    (rhs is transformed to Chebyshev space in place by the reference)."""
    rhs = np.array(rhs, dtype=np.complex128, order="F")
    my, mz, nm = rhs.shape
    sol = np.zeros_like(rhs, order="F")
    xalp = np.ascontiguousarray(xalp, dtype=np.float64)
    rc = lib().orc_helm3d_shen(_p(rhs), _p(sol), my, mz, ib, ib + nm - 1, _p(xalp), float(alambda),
                               C.byref(shen._s), int(nthreads))
    if rc:
        raise ValueError("orc_helm3d_shen: grid %dx%d does not match the set-up %d" % (my, mz, shen.m))
    return sol, rhs


def helm3d_temp(rhs, ydir, zdir, alambda, xalp, ib=0, bcy=None, bcz=None, nthreads=1):
    """helm3d_temp on a complex (my,mz,nmodes) field; bcy (mz,2,nmodes),
    bcz (my,2,nmodes) real wall values or None.  Returns the solution."""
    rhs = np.asfortranarray(rhs, dtype=np.complex128)
    my, mz, nm = rhs.shape
    sol = np.zeros_like(rhs, order="F")
    xalp = np.ascontiguousarray(xalp, dtype=np.float64)
    by = None if bcy is None else np.asfortranarray(bcy, dtype=np.float64)
    bz = None if bcz is None else np.asfortranarray(bcz, dtype=np.float64)
    lib().orc_helm3d_temp(_p(rhs), _p(sol), my, mz, ib, ib + nm - 1, _p(xalp), float(alambda),
                          C.byref(ydir._s), C.byref(zdir._s), _p(by), _p(bz), int(nthreads))
    return sol


def solvediag(U, ops, bound, xlambda):
    """solvediag on one real (my,mz) plane; returns a new array."""
    U = np.asfortranarray(U, dtype=np.float64).copy(order="F")
    r = lib().orc_solvediag(_p(U), C.byref(ops._s), bound.encode(), float(xlambda))
    if r:
        raise ValueError("solvediag: bad bound")
    return U


def helm3d(rhs, ops, bound, alambda, xalp, ib=0, nthreads=1):
    """helm3d on a complex (my,mz,nmodes) field.  Returns (sol, rhs_after)
    where rhs_after carries helm3d's in-place wall zeroing for bound='d'."""
    rhs = np.asfortranarray(rhs, dtype=np.complex128).copy(order="F")
    my, mz, nm = rhs.shape
    sol = np.zeros_like(rhs, order="F")
    xalp = np.ascontiguousarray(xalp, dtype=np.float64)
    assert xalp.shape == (nm,)
    r = lib().orc_helm3d(_p(rhs), _p(sol), my, mz, ib, ib + nm - 1, _p(xalp),
                         bound.encode(), float(alambda), C.byref(ops._s), int(nthreads))
    if r:
        raise ValueError("helm3d failed (%d)" % r)
    return sol, rhs


def transyz(f, cdir, iopt):
    f = np.asfortranarray(f, dtype=np.complex128).copy(order="F")
    my, mz, nm = f.shape
    lib().orc_transyz(_p(f), my, mz, nm, cdir.encode(), int(iopt))
    return f


def cheb_interp(f, my, mz):
    """cheb_interp(myr,mzr,tmp1,my,mz,tmpo1), src/chebyshev.f90:725-765, on
    every mode of a complex (myr, mzr, M) field: each plane's Chebyshev
    coefficients (transyz_plane_fou -1), the first min(20, myr) x min(20,
    mzr) of them summed at the nodes of the (my, mz) grid, T_k(y2) =
    cos(k acos(y2)) with y2 = -dglc(-1, 1) (src/chebyshev.f90:429-456)."""
    c = transyz(transyz(f, "y", -1), "z", -1)
    myr, mzr, M = c.shape
    K, L = min(20, myr), min(20, mzr)
    pi = 4.0 * np.arctan(1.0)
    y2 = -(-np.cos(np.arange(my) * (pi / (my - 1))))
    z2 = -(-np.cos(np.arange(mz) * (pi / (mz - 1))))
    ty = np.cos(np.outer(np.arccos(y2), np.arange(K)))      # (my, K)
    tz = np.cos(np.outer(np.arccos(z2), np.arange(L)))      # (mz, L)
    out = np.zeros((my, mz, M), dtype=np.complex128, order="F")
    for m in range(M):
        out[:, :, m] = ty @ c[:K, :L, m] @ tz.T
    return out


def transyz_plane(f, iopt):
    f = np.asfortranarray(f, dtype=np.float64).copy(order="F")
    my, mz = f.shape
    lib().orc_transyz_plane(_p(f), my, mz, int(iopt))
    return f


def derivyz(u, cdir, ider, scal=1.0, what="n", du=None, aspect=1.0):
    u = np.asfortranarray(u, dtype=np.complex128)
    my, mz, nm = u.shape
    du = np.zeros_like(u, order="F") if du is None else np.asfortranarray(du).copy(order="F")
    lib().orc_derivyz(_p(u), _p(du), my, mz, nm, cdir.encode(), int(ider), float(scal),
                      what.encode(), float(aspect))
    return du


def cheb2_integral(u, aspect=1.0):
    u = np.asfortranarray(u, dtype=np.float64)
    return lib().orc_cheb2_integral(_p(u), u.shape[0], u.shape[1], float(aspect))


def cxyz2yzx(phys):
    """phys (0:mx1, my, nz) complex -> (my, nz, 0:mx1)."""
    phys = np.asfortranarray(phys, dtype=np.complex128)
    nm, my, nz = phys.shape
    out = np.zeros((my, nz, nm), dtype=np.complex128, order="F")
    lib().orc_cxyz2yzx(_p(phys), _p(out), nm, my, nz)
    return out


def cyzx2xyz(phys2):
    """phys2 (my, nz, 0:mx1) complex -> (0:mx1, my, nz)."""
    phys2 = np.asfortranarray(phys2, dtype=np.complex128)
    my, nz, nm = phys2.shape
    out = np.zeros((nm, my, nz), dtype=np.complex128, order="F")
    lib().orc_cyzx2xyz(_p(out), _p(phys2), nm, my, nz)
    return out


def set_blas_threads(n):
    lib().orc_set_blas_threads(int(n))


__all__ = ["Ops", "Dir", "Shen", "Pois", "solvepois", "cheb_interp", "precomp_mass_flow", "impose_mass_flow", "solveshen", "helm3d_shen", "helm3d_temp", "solvediag", "helm3d", "transyz", "transyz_plane", "derivyz",
           "cheb2_integral", "cxyz2yzx", "cyzx2xyz", "set_blas_threads", "lib"]
_ = os


# ---- DNS time step around the solve (duct_oracle_dns.c) -------------------
class _DnsStats(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in ("mean", "prod", "ppb", "spec")] + [
        ("stress4", C.c_double * 4), ("energy", C.c_double * 3), ("energy2", C.c_double * 3),
        ("nstat", C.c_int), ("om2", C.POINTER(C.c_double)), ("omg", C.c_double * 16),
        ("cfl2", C.c_double * 2)]


def _dns_sigs(L):
    P, I, D = C.c_void_p, C.c_int, C.c_double
    L.orc_fourx.argtypes = [P, P, I, I, I, I, I]
    L.orc_derivx.argtypes = [P, P, I, I, I, P, I, D, C.c_char]
    L.orc_advection3d.argtypes = [P, P, P, P, P, P, I, I, I, I, P, D, P]
    L.orc_laplacian3d.argtypes = [P, P, I, I, I, P, D, D, C.c_char]
    L.orc_vorticity.argtypes = [P, P, P, P, P, I, I, I, P, D, I]
    L.orc_grad3d.argtypes = [P, P, P, P, I, I, I, P, D, D, C.c_char]
    L.orc_div3d.argtypes = [P, P, P, P, I, I, I, P, D, D]
    L.orc_update_uvwp.argtypes = [P, P, P, P, P, P, I, I, I, P, D, D, D, D, D]
    L.orc_max_3din.argtypes = [P, I, I, I]
    L.orc_max_3din.restype = D
    L.orc_wallstressx.argtypes = [P, I, I, D, P]
    L.orc_energy_fou.argtypes = [P, I, I, I, D, C.POINTER(D), C.POINTER(D)]
    L.orc_statistics_fou.argtypes = [P, P, P, P, I, I, I, P, P, P]
    L.orc_rk_coefficients.argtypes = [P, P, P, P]
    L.orc_dns_substep.argtypes = [P, P, P, P, P, P, P, P, P, P, I, I, I, I, P, D, D, D, I, C.POINTER(_Ops), I,
                                  D, P, P, D, C.POINTER(_DnsStats), I, P]
    L.orc_dns_substep.restype = D


def _dlib():
    L = lib()
    if not getattr(L, "_dns_ready", False):
        _dns_sigs(L)
        L._dns_ready = True
    return L


def _cf(a):
    return np.array(a, dtype=np.complex128, order="F")


def fourx(fou=None, phys=None, mgalx=None, iopt=1):
    """fourx (src/fourier.F:1-68): iopt >= 0 takes a z-cut complex
    (M, my, nz) array and returns phys (mgalx+2, my, nz); iopt < 0 the
    inverse (returns the z-cut (M, my, nz) array, M given by fou's shape)."""
    L = _dlib()
    if iopt >= 0:
        fou = _cf(fou)
        M, my, nz = fou.shape
        out = np.zeros((mgalx + 2, my, nz), order="F")
        L.orc_fourx(_p(fou), _p(out), M - 1, mgalx, my, nz, int(iopt))
        return out
    phys = np.asfortranarray(phys, dtype=np.float64)
    n2, my, nz = phys.shape
    out = np.zeros(fou.shape if fou is not None else (None,), dtype=np.complex128, order="F")
    L.orc_fourx(_p(out), _p(phys), out.shape[0] - 1, n2 - 2, my, nz, int(iopt))
    return out


def derivx(u, xalp, ider, scal=1.0, what="n", du=None):
    L = _dlib()
    u = _cf(u)
    my, mz, M = u.shape
    du = np.zeros_like(u, order="F") if du is None else _cf(du)
    L.orc_derivx(_p(u), _p(du), my, mz, M, _p(np.ascontiguousarray(xalp, dtype=np.float64)), int(ider),
                 float(scal), what.encode())
    return du


def advection3d(u, v, w, mgalx, xalp, aspect=1.0, stats=False):
    """advection3d (src/operators.F:9-276) on x-cut fields; returns
    (adv1, adv2, adv3) and, with stats, the six product x-means
    (uub, vvb, wwb, uvb, uwb, vwb) as a (6, my, mz) array."""
    L = _dlib()
    u, v, w = _cf(u), _cf(v), _cf(w)
    my, mz, M = u.shape
    a1, a2, a3 = (np.zeros_like(u, order="F") for _ in range(3))
    st = np.zeros((my, mz, 6), order="F") if stats else None
    L.orc_advection3d(_p(u), _p(v), _p(w), _p(a1), _p(a2), _p(a3), my, mz, M, int(mgalx),
                      _p(np.ascontiguousarray(xalp, dtype=np.float64)), float(aspect), _p(st))
    if stats:
        return a1, a2, a3, np.moveaxis(st, 2, 0)
    return a1, a2, a3


def vorticity(u, v, w, xalp, iflag, aspect=1.0):
    """vorticity (src/operators.F:810-905), component iflag (1, 2, 3); the
    inputs are copied (the reference's round trips change them in place)."""
    L = _dlib()
    u, v, w = (np.array(_cf(f), order="F") for f in (u, v, w))
    my, mz, M = u.shape
    vort, tmp = np.zeros_like(u, order="F"), np.zeros_like(u, order="F")
    L.orc_vorticity(_p(u), _p(v), _p(w), _p(vort), _p(tmp), my, mz, M,
                    _p(np.ascontiguousarray(xalp, dtype=np.float64)), float(aspect), int(iflag))
    return vort


def laplacian3d(u, xalp, scal, what="n", flap=None, aspect=1.0):
    """Returns (flap, u_after): u is transformed in place and back."""
    L = _dlib()
    u = _cf(u)
    my, mz, M = u.shape
    flap = np.zeros_like(u, order="F") if flap is None else _cf(flap)
    L.orc_laplacian3d(_p(u), _p(flap), my, mz, M, _p(np.ascontiguousarray(xalp, dtype=np.float64)),
                      float(aspect), float(scal), what.encode())
    return flap, u


def grad3d(u, xalp, scal, what="n", out=None, aspect=1.0):
    L = _dlib()
    u = _cf(u)
    my, mz, M = u.shape
    dx, dy, dz = (np.zeros_like(u, order="F") for _ in range(3)) if out is None else (_cf(o) for o in out)
    L.orc_grad3d(_p(u), _p(dx), _p(dy), _p(dz), my, mz, M, _p(np.ascontiguousarray(xalp, dtype=np.float64)),
                 float(aspect), float(scal), what.encode())
    return dx, dy, dz


def div3d(u, v, w, xalp, scal, aspect=1.0):
    L = _dlib()
    u, v, w = _cf(u), _cf(v), _cf(w)
    my, mz, M = u.shape
    d = np.zeros_like(u, order="F")
    L.orc_div3d(_p(u), _p(v), _p(w), _p(d), my, mz, M, _p(np.ascontiguousarray(xalp, dtype=np.float64)),
                float(aspect), float(scal))
    return d


def update_uvwp(u, v, w, p, phi, xalp, akk, bkk, dt, fnu, aspect=1.0):
    """Returns (u, v, w, p, phi_after, rhsphi)."""
    L = _dlib()
    u, v, w, p, phi = _cf(u), _cf(v), _cf(w), _cf(p), _cf(phi)
    my, mz, M = u.shape
    rhs = np.zeros_like(u, order="F")
    L.orc_update_uvwp(_p(u), _p(v), _p(w), _p(p), _p(phi), _p(rhs), my, mz, M,
                      _p(np.ascontiguousarray(xalp, dtype=np.float64)), float(aspect), float(akk), float(bkk),
                      float(dt), float(fnu))
    return u, v, w, p, phi, rhs


def max_3din(u):
    u = _cf(u)
    return _dlib().orc_max_3din(_p(u), *u.shape)


def wallstressx(u, aspect=1.0):
    u = _cf(u)
    out = np.zeros(4)
    _dlib().orc_wallstressx(_p(u), u.shape[0], u.shape[1], float(aspect), _p(out))
    return out


def energy_fou(u, aspect=1.0):
    u = _cf(u)
    e, e2 = C.c_double(), C.c_double()
    _dlib().orc_energy_fou(_p(u), *u.shape, float(aspect), C.byref(e), C.byref(e2))
    return e.value, e2.value


def rk_coefficients():
    a, b, g, r = (np.zeros(3) for _ in range(4))
    _dlib().orc_rk_coefficients(_p(a), _p(b), _p(g), _p(r))
    return a, b, g, r


class Dns:
    """The RK3/CN time step of src/main1.f90:384-723 (square duct, no
    temperature, DT_FIXED) on x-cut complex (my, my, M) fields, with the
    statistics of src/operators.F gathered at the first substep of a step.
    cmassflow True: the flow rate of the initial u is held
    (impose_mass_flow after every substep); else the mean pressure gradient
    dpdx drives the flow."""

    def __init__(self, u, v, w, p, mgalx, alp, fnu, dt, cmassflow=True, dpdx=0.0, aspect=1.0, nthreads=1):
        L = _dlib()
        self.u, self.v, self.w, self.p = (_cf(f) for f in (u, v, w, p))
        my, mz, M = self.u.shape
        assert my == mz
        self.my, self.M, self.mgalx = my, M, int(mgalx)
        self.xalp = alp * np.arange(M, dtype=np.float64)
        self.fnu, self.dt, self.aspect, self.nthreads = float(fnu), float(dt), float(aspect), int(nthreads)
        self.adv = [np.zeros_like(self.u, order="F") for _ in range(3)]
        self.h = [np.zeros_like(self.u, order="F") for _ in range(3)]
        self.ops = Ops(my)
        self.cmassflow, self.dpdx = bool(cmassflow), float(dpdx)
        a, b, g, r = rk_coefficients()
        self.premassfu, self.premassf = precomp_mass_flow(self.ops, self.dt, b, self.fnu, aspect)
        _, self.csum, _ = impose_mass_flow(self.u, 0.0, 1, self.premassfu, self.premassf, 0, aspect)
        self.stats_mean = np.zeros((my, mz, 4), order="F")
        self.stats_prod = np.zeros((my, mz, 6), order="F")
        self.stats_ppb = np.zeros((my, mz), order="F")
        self.stats_spec = np.zeros((M, 7, 4), order="F")
        self._st = _DnsStats()
        self._st.mean = self.stats_mean.ctypes.data_as(C.POINTER(C.c_double))
        self._st.prod = self.stats_prod.ctypes.data_as(C.POINTER(C.c_double))
        self._st.ppb = self.stats_ppb.ctypes.data_as(C.POINTER(C.c_double))
        self._st.spec = self.stats_spec.ctypes.data_as(C.POINTER(C.c_double))
        self.stats_om2 = np.zeros((my, mz, 3), order="F")
        self._st.om2 = self.stats_om2.ctypes.data_as(C.POINTER(C.c_double))
        self.history = []
        self.divmax = None
        self.force = None

    def set_forcing(self, f=None):
        """Body force (f1, f2, f3), h += (akk+bkk) f in every substep; None removes it."""
        self.force = None if f is None else np.asfortranarray(np.stack([_cf(x) for x in f], axis=3))

    def substep(self, krk, stats=False):
        L = _dlib()
        self.divmax = L.orc_dns_substep(
            _p(self.u), _p(self.v), _p(self.w), _p(self.p), _p(self.adv[0]), _p(self.adv[1]), _p(self.adv[2]),
            _p(self.h[0]), _p(self.h[1]), _p(self.h[2]), self.my, self.my, self.M, self.mgalx, _p(self.xalp),
            self.aspect, self.fnu, self.dt, int(krk), C.byref(self.ops._s), int(self.cmassflow), float(self.csum),
            _p(self.premassfu), _p(self.premassf), self.dpdx, C.byref(self._st) if stats else None,
            self.nthreads, None if self.force is None else _p(self.force))
        if stats and krk == 1:
            self.history.append(dict(stress4=list(self._st.stress4), energy=list(self._st.energy),
                                     energy2=list(self._st.energy2), omg=list(self._st.omg),
                                     remx=self._st.cfl2[0], slip=self._st.cfl2[1]))
        return self.divmax

    def step(self, stats=False):
        for krk in (1, 2, 3):
            self.substep(krk, stats=stats)
        return self.divmax

    def statistics_omg(self):
        """The vorticity diagnostics (src/main1.f90:453-466): om2 (3,my,mz)
        summed over the recorded steps, hist (nstep,16) one row per step."""
        return dict(om2=np.moveaxis(self.stats_om2, 2, 0).copy(),
                    hist=np.array([h["omg"] for h in self.history]).reshape(-1, 16))

    def statistics(self):
        """Accumulated statistics, each summed over the recorded steps:
        dict(nstat, mean (4,my,mz), prod (6,my,mz), ppb (my,mz), spec (4,7,M))."""
        return dict(nstat=self._st.nstat, mean=np.moveaxis(self.stats_mean, 2, 0).copy(),
                    prod=np.moveaxis(self.stats_prod, 2, 0).copy(), ppb=self.stats_ppb.copy(),
                    spec=np.transpose(self.stats_spec, (2, 1, 0)).copy())
