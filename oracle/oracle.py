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


__all__ = ["Ops", "Dir", "Shen", "Pois", "solvepois", "precomp_mass_flow", "impose_mass_flow", "solveshen", "helm3d_shen", "helm3d_temp", "solvediag", "helm3d", "transyz", "transyz_plane", "derivyz",
           "cheb2_integral", "cxyz2yzx", "cyzx2xyz", "set_blas_threads", "lib"]
_ = os
