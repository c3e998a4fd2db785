"""duct_b200 -- B200 (sm_100a) implementation of the duct per-Fourier-mode
2D Helmholtz/Poisson diagonalisation solve behind a C-ABI.

The product is ``duct_b200/lib/libductgpu.so`` (C-ABI declared in
``include/ductgpu.h``).  This module is a thin ctypes mirror of that ABI for
Python callers, tests and the benchmark; it does no numerics of its own and
there is no CPU fallback: if the library is missing, importing raises.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libductgpu.so")

OK, EARG, ESTATE, ECUDA, ESOLVER, ENONFINITE, ETIMEOUT, EALLOC = range(8)
PREC_FP64, PREC_MIXED, PREC_INT8 = 0, 1, 2
PASS_STAGED, PASS_REGISTER, PASS_STAGED16, PASS_PERSIST, PASS_PARITY, PASS_PARITY_QUEUE = 0, 1, 2, 3, 4, 5
GAUGE_POINT, GAUGE_MEAN = 0, 1

EXPORTS = [
    "ductgpu_create", "ductgpu_destroy", "ductgpu_last_error", "ductgpu_set_stream",
    "ductgpu_get_stream", "ductgpu_synchronize", "ductgpu_selftest_wait_timeout", "ductgpu_pseudomat",
    "ductgpu_get_operators", "ductgpu_set_operators", "ductgpu_set_gauge",
    "ductgpu_helm3d", "ductgpu_solve_fields_dev", "ductgpu_device_alloc",
    "ductgpu_device_free", "ductgpu_host_alloc", "ductgpu_host_free", "ductgpu_copy",
    "ductgpu_event_record", "ductgpu_event_elapsed", "ductgpu_launch_count",
    "ductgpu_profile_enable", "ductgpu_profile_reset", "ductgpu_profile_read",
    "ductgpu_transyz_dev", "ductgpu_transyz", "ductgpu_derivyz_dev", "ductgpu_derivyz",
    "ductgpu_cxyz2yzx_dev", "ductgpu_cyzx2xyz_dev", "ductgpu_chx2z_dev", "ductgpu_chz2x_dev",
    "ductgpu_set_refinement", "ductgpu_pseudomat_temp", "ductgpu_helm3d_temp",
    "ductgpu_solve_rect_fields_dev", "ductgpu_graph_create", "ductgpu_graph_launch",
    "ductgpu_graph_destroy", "transpose_gpu_", "mat_invdiag_gpu_",
    "ductgpu_preshen", "ductgpu_helm3d_shen", "ductgpu_solve_shen_fields_dev",
    "ductgpu_solve_fields_dev_noalloc", "ductgpu_precomp_mass_flow",
    "ductgpu_impose_mass_flow_dev", "ductgpu_impose_mass_flow",
    "ductgpu_solve_adjoint_fields_dev", "ductgpu_helm3d_adjoint",
    "ductgpu_pseudopois", "ductgpu_solvepois", "ductgpu_solve_pois_fields_dev",
    "ductgpu_set_pass_kernel", "ductgpu_autotune", "ductgpu_helm3d_batch",
    "ductgpu_pseudomat_ex", "ductgpu_set_gauge_point", "ductgpu_get_fold",
    "ductgpu_derivx_dev", "ductgpu_laplacian3d_dev", "ductgpu_grad3d_dev", "ductgpu_div3d_dev",
    "ductgpu_update_uvwp_dev", "ductgpu_advection3d_dev", "ductgpu_max_3din_dev",
    "ductgpu_wallstressx_dev", "ductgpu_energy_fou_dev", "ductgpu_statistics_fou_dev",
    "ductgpu_dns_create", "ductgpu_dns_destroy", "ductgpu_dns_set_fields", "ductgpu_dns_get_fields",
    "ductgpu_dns_field", "ductgpu_dns_set_graphs", "ductgpu_dns_substep", "ductgpu_dns_steps",
    "ductgpu_dns_statistics", "ductgpu_profile_bytes", "ductgpu_profile_flops", "ductgpu_cheb_deriv_matrix", "ductgpu_dns_set_forcing",
    "ductgpu_dns_wallstress_after", "ductgpu_dns_grad_wallstress", "ductgpu_set_rect_fold",
    "ductgpu_set_line_kernel", "ductgpu_uvwp_filename", "ductgpu_save_4fields_fou_hdf5_dev",
    "ductgpu_read_hdf5_header", "ductgpu_read_4fields_fou_hdf5_dev", "ductgpu_dns_save_hdf5",
    "ductgpu_dns_load_hdf5", "ductgpu_vorticity_dev", "ductgpu_dns_statistics_omg", "ductgpu_dns_cfl",
    "ductgpu_dns_write_statistics_hdf5", "ductgpu_statistics_filename",
]
SETUP_NO_EIGEN = 1
(K_PASS_FP64, K_NEUMANN, K_WALLS, K_MIXED_GEMM, K_RESIDUAL, K_TRANSFORM, K_TRANSPOSE, K_OTHER, K_LINES,
 K_ADVECTION, K_STATS) = range(11)
K_COUNT = 11


class RectField(C.Structure):
    """ductgpu_rect_field of include/ductgpu.h."""
    _fields_ = [("rhs", C.c_void_p), ("sol", C.c_void_p), ("xalp", C.c_void_p), ("bcy", C.c_void_p),
                ("bcz", C.c_void_p), ("alambda", C.c_double), ("ib", C.c_int), ("nmodes", C.c_int),
                ("slot", C.c_int)]


class Field(C.Structure):
    """ductgpu_field of include/ductgpu.h."""
    _fields_ = [("rhs", C.c_void_p), ("sol", C.c_void_p), ("xalp", C.c_void_p),
                ("alambda", C.c_double), ("ib", C.c_int), ("nmodes", C.c_int),
                ("bound", C.c_char)]


class H5Header(C.Structure):
    """ductgpu_h5_header of include/ductgpu.h (writeheader_hdf5's scalars)."""
    _fields_ = [("nparams", C.c_int), ("numerop", C.c_int), ("mgalx", C.c_int), ("my", C.c_int),
                ("mz", C.c_int), ("mx1", C.c_int), ("alp", C.c_double), ("aspect", C.c_double),
                ("time", C.c_double), ("fnu", C.c_double), ("cfl", C.c_double), ("dtfixed", C.c_double),
                ("cmassflow", C.c_double), ("slip", C.c_double), ("divergence", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

    @classmethod
    def from_dict(cls, d):
        h = cls()
        for k, _ in cls._fields_:
            if k in d:
                setattr(h, k, d[k])
        return h


_lib = None


def lib():
    """Load libductgpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libductgpu.so is not built (run duct_b200/build.py): %s" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        P, I, D = C.c_void_p, C.c_int, C.c_double
        sig = {
            "ductgpu_create": [I, C.POINTER(P)],
            "ductgpu_destroy": [P],
            "ductgpu_last_error": [P, C.c_char_p, I],
            "ductgpu_set_stream": [P, P],
            "ductgpu_get_stream": [P],
            "ductgpu_synchronize": [P],
            "ductgpu_selftest_wait_timeout": [P, C.c_uint],
            "ductgpu_pseudomat": [P, I, I],
            "ductgpu_pseudomat_ex": [P, I, I, I],
            "ductgpu_set_gauge_point": [P, I],
            "ductgpu_get_fold": [P, C.c_char, C.POINTER(I)],
            "ductgpu_get_operators": [P, C.c_char, P, P, P, C.POINTER(I)],
            "ductgpu_set_operators": [P, C.c_char, P, P, P, I],
            "ductgpu_set_gauge": [P, I],
            "ductgpu_helm3d": [P, P, P, I, C.c_char, D, I, I, I, I, P, I],
            "ductgpu_solve_fields_dev": [P, C.POINTER(Field), I, I],
            "ductgpu_device_alloc": [P, C.c_size_t, C.POINTER(P)],
            "ductgpu_device_free": [P, P],
            "ductgpu_host_alloc": [P, C.c_size_t, C.POINTER(P)],
            "ductgpu_host_free": [P, P],
            "ductgpu_copy": [P, P, P, C.c_size_t, I],
            "ductgpu_event_record": [P, I],
            "ductgpu_event_elapsed": [P, I, I, C.POINTER(C.c_float)],
            "ductgpu_launch_count": [P],
            "ductgpu_profile_enable": [P, I],
            "ductgpu_profile_reset": [P],
            "ductgpu_profile_read": [P, I, C.POINTER(C.c_double), C.POINTER(C.c_longlong)],
            "ductgpu_transyz_dev": [P, P, I, I, I, C.c_char, I],
            "ductgpu_transyz": [P, P, I, I, I, C.c_char, I],
            "ductgpu_derivyz_dev": [P, P, P, I, I, I, C.c_char, I, D, C.c_char, D],
            "ductgpu_derivyz": [P, P, P, I, I, I, C.c_char, I, D, C.c_char, D],
            "ductgpu_cxyz2yzx_dev": [P, P, P, I, I, I],
            "ductgpu_cyzx2xyz_dev": [P, P, P, I, I, I],
            "ductgpu_chx2z_dev": [P, P, P, I, I, I],
            "ductgpu_chz2x_dev": [P, P, P, I, I, I],
            "ductgpu_set_refinement": [P, I],
            "ductgpu_pseudomat_temp": [P, I, I, I, D, D, C.c_char, C.c_char, C.c_char, C.c_char],
            "ductgpu_helm3d_temp": [P, P, P, I, D, D, D, I, I, I, I, P, P, P, C.c_char, C.c_char,
                                    C.c_char, C.c_char],
            "ductgpu_solve_rect_fields_dev": [P, C.POINTER(RectField), I],
            "ductgpu_graph_create": [P, I, P, I, I, C.POINTER(I)],
            "ductgpu_preshen": [P, I, C.c_char],
            "ductgpu_helm3d_shen": [P, P, P, I, C.c_char, D, I, I, I, I, P],
            "ductgpu_solve_shen_fields_dev": [P, C.POINTER(Field), I],
            "ductgpu_solve_fields_dev_noalloc": [P, C.POINTER(Field), I],
            "ductgpu_precomp_mass_flow": [P, D, P, I, D, D, P, P],
            "ductgpu_impose_mass_flow_dev": [P, C.POINTER(D), I, P, I],
            "ductgpu_impose_mass_flow": [P, C.POINTER(D), I, P, I],
            "ductgpu_solve_adjoint_fields_dev": [P, C.POINTER(Field), I],
            "ductgpu_helm3d_adjoint": [P, P, P, C.c_char, D, I, I, I, I, P],
            "ductgpu_pseudopois": [P, I],
            "ductgpu_set_pass_kernel": [P, I, I],
            "ductgpu_autotune": [P, C.POINTER(Field), I, I, C.POINTER(I)],
            "ductgpu_helm3d_batch": [P, I, P, P, C.c_char_p, P, I, I, I, I, P, I],
            "ductgpu_solvepois": [P, P, D, I],
            "ductgpu_solve_pois_fields_dev": [P, C.POINTER(Field), I],
            "ductgpu_graph_launch": [P, I],
            "ductgpu_derivx_dev": [P, P, P, I, I, I, P, I, D, C.c_char],
            "ductgpu_laplacian3d_dev": [P, P, P, I, I, I, P, D, D, C.c_char],
            "ductgpu_grad3d_dev": [P, P, P, P, P, I, I, I, P, D, D, C.c_char],
            "ductgpu_div3d_dev": [P, P, P, P, P, I, I, I, P, D, D],
            "ductgpu_update_uvwp_dev": [P, P, P, P, P, P, I, I, I, P, D, D, D, D, D],
            "ductgpu_advection3d_dev": [P, P, P, P, P, P, P, P, I, I, I, I, P, D, P],
            "ductgpu_max_3din_dev": [P, P, I, I, I, C.POINTER(D)],
            "ductgpu_wallstressx_dev": [P, P, I, I, D, P],
            "ductgpu_energy_fou_dev": [P, P, I, I, I, D, C.POINTER(D), C.POINTER(D)],
            "ductgpu_statistics_fou_dev": [P, P, P, P, P, I, I, I, P, P, P],
            "ductgpu_dns_create": [P, I, D, D, D, D, I, D, I, I, C.POINTER(P)],
            "ductgpu_dns_destroy": [P],
            "ductgpu_dns_set_fields": [P, P, P, P, P],
            "ductgpu_dns_get_fields": [P, P, P, P, P],
            "ductgpu_dns_field": [P, I, C.POINTER(P)],
            "ductgpu_dns_set_graphs": [P, I],
            "ductgpu_dns_substep": [P, I, I],
            "ductgpu_dns_steps": [P, I, I],
            "ductgpu_dns_statistics": [P, P, P, P, P, P, C.POINTER(I), C.POINTER(I), P],
            "ductgpu_profile_bytes": [P, I, C.POINTER(D)],
            "ductgpu_profile_flops": [P, I, C.POINTER(D)],
            "ductgpu_cheb_deriv_matrix": [I, I, C.POINTER(D)],
            "ductgpu_dns_set_forcing": [P, P, P, P],
            "ductgpu_set_rect_fold": [P, I],
            "ductgpu_set_line_kernel": [P, I],
            "ductgpu_dns_wallstress_after": [P, I, C.POINTER(D)],
            "ductgpu_dns_grad_wallstress": [P, C.POINTER(D), P],
            "ductgpu_graph_destroy": [P, I],
            "ductgpu_uvwp_filename": [C.c_char_p, I, C.c_char_p, I],
            "ductgpu_save_4fields_fou_hdf5_dev": [P, C.c_char_p, P, P, P, P, C.POINTER(H5Header)],
            "ductgpu_read_hdf5_header": [P, C.c_char_p, C.POINTER(H5Header)],
            "ductgpu_read_4fields_fou_hdf5_dev": [P, C.c_char_p, P, P, P, P, I, I, I, C.POINTER(H5Header)],
            "ductgpu_dns_save_hdf5": [P, C.c_char_p, D, D, D],
            "ductgpu_dns_load_hdf5": [P, C.c_char_p, C.POINTER(D)],
            "ductgpu_vorticity_dev": [P, P, P, P, P, I, I, I, P, D, I],
            "ductgpu_dns_statistics_omg": [P, P, P, C.POINTER(I)],
            "ductgpu_dns_cfl": [P, C.POINTER(D), C.POINTER(D), C.POINTER(D)],
            "ductgpu_dns_write_statistics_hdf5": [P, C.c_char_p, D, D],
            "ductgpu_statistics_filename": [C.c_char_p, C.c_char_p, I],
            "transpose_gpu_": [P, C.POINTER(I), C.POINTER(I), C.POINTER(D), C.POINTER(C.c_size_t),
                               C.POINTER(C.c_size_t)],
            "mat_invdiag_gpu_": [P, C.POINTER(I), C.POINTER(I), C.POINTER(D), C.POINTER(C.c_size_t),
                                 C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = I
        L.ductgpu_get_stream.restype = P
        L.ductgpu_launch_count.restype = C.c_longlong
        _lib = L
    return _lib


def cheb_deriv_matrix(n, order):
    """The n x n real matrix of the reference's derivative chain along one
    Chebyshev direction (transyz -1, derivyz of this order, transyz +1), as
    the tensor-core line kernel applies it; host only (no GPU needed)."""
    out = np.zeros((n, n), dtype=np.float64, order="F")
    rc = lib().ductgpu_cheb_deriv_matrix(int(n), int(order), out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc:
        raise DuctGPUError(rc, "cheb_deriv_matrix: n=%d order=%d" % (n, order))
    return out


def uvwp_filename(fuvwpout, iimag):
    """The reference's field file name: prefix (up to its first blank) +
    'uvwp_' + iimag as i4.4 + '.h5' (ductgpu_uvwp_filename)."""
    buf = C.create_string_buffer(4096)
    rc = lib().ductgpu_uvwp_filename(os.fsencode(fuvwpout), int(iimag), buf, 4096)
    if rc:
        raise DuctGPUError(rc, "uvwp_filename")
    return buf.value.decode()


def statistics_filename(fuvwpout):
    """The reference's statistics file name: prefix + 'statistics_NNNN.h5'
    with the first NNNN whose file does not exist yet."""
    buf = C.create_string_buffer(4096)
    rc = lib().ductgpu_statistics_filename(os.fsencode(fuvwpout), buf, 4096)
    if rc:
        raise DuctGPUError(rc, "statistics_filename")
    return buf.value.decode()


def read_hdf5_header(filename):
    """readheader_hdf5 of a uvwp_NNNN.h5 file, as a dict (no GPU needed)."""
    h = H5Header()
    rc = lib().ductgpu_read_hdf5_header(None, os.fsencode(filename), C.byref(h))
    if rc:
        raise DuctGPUError(rc, "read_hdf5_header(%s) failed" % filename)
    return h.as_dict()


def fortran_e15_8(x):
    """A double as Fortran's e15.8 edit descriptor writes it
    (" 0.12345678E+01"; the exponent in two digits up to 99)."""
    import math
    x = float(x)
    if x == 0.0 or not math.isfinite(x):
        return " 0.00000000E+00" if x == 0.0 else ("%15s" % x)
    e = math.floor(math.log10(abs(x))) + 1
    m = "%.8f" % (abs(x) / 10.0 ** e)
    if m.startswith("1"):          # rounding reached 1.0: next decade
        e += 1
        m = "%.8f" % (abs(x) / 10.0 ** e)
    if m.startswith("0.0"):        # below 0.1 after rounding down the power
        e -= 1
        m = "%.8f" % (abs(x) / 10.0 ** e)
    exp = ("E+%02d" if e >= 0 else "E-%02d") % abs(e)
    return ("-" if x < 0 else " ") + m + exp


def ener_line(time, hist_row, omg_row):
    """The reference's per-step log line (src/main1.f90:471-486, format 111:
    'ENER: ', 38 values as e15.8 each followed by a blank) from one row of
    Dns.statistics()['hist'] (stress4[4], energy of u, v, w, the same with
    mode 0) and the matching row of Dns.statistics_omg()['hist'].  The
    temperature columns and energi (not computed by the reference either)
    are 0."""
    st, en, en2 = list(hist_row[0:4]), list(hist_row[4:7]), list(hist_row[7:10])
    ox4, oxb4, om, omb = list(omg_row[0:5]), list(omg_row[5:10]), list(omg_row[10:13]), list(omg_row[13:16])
    import math
    vals = ([time, sum(st), sum(en)] + en + [0.0, math.sqrt(sum(ox4))] + st + ox4[:4] + oxb4[:4] +
            [ox4[4], oxb4[4], 0.0] + en2 + [0.0] + [0.0] * 4 + om + omb + [0.0])
    assert len(vals) == 38
    return "ENER: " + "".join(fortran_e15_8(v) + " " for v in vals)


class DuctGPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("ductgpu status %d: %s" % (code, msg))
        self.code = code


def _ptr(a):
    if isinstance(a, DeviceArray):
        return C.c_void_p(a.ptr)
    if a is None:
        return None
    assert a.flags.f_contiguous or a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


class DeviceArray:
    """Device buffer owned through the library's allocation helpers."""

    def __init__(self, ctx, shape, dtype=np.complex128):
        self.ctx, self.shape, self.dtype = ctx, tuple(shape), np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = C.c_void_p()
        ctx._check(lib().ductgpu_device_alloc(ctx.h, self.nbytes, C.byref(p)))
        self.ptr = p.value

    def upload(self, host):
        host = np.asfortranarray(host, dtype=self.dtype)
        assert host.nbytes == self.nbytes
        self.ctx._check(lib().ductgpu_copy(self.ctx.h, C.c_void_p(self.ptr), _ptr(host), self.nbytes, 1))
        self.ctx.synchronize()

    def download(self):
        out = np.empty(self.shape, dtype=self.dtype, order="F")
        self.ctx._check(lib().ductgpu_copy(self.ctx.h, _ptr(out), C.c_void_p(self.ptr), self.nbytes, 2))
        self.ctx.synchronize()
        return out

    def free(self):
        if self.ptr:
            lib().ductgpu_device_free(self.ctx.h, C.c_void_p(self.ptr))
            self.ptr = None


class Context:
    """One ductgpu context (device + stream + operators)."""

    def __init__(self, device=0):
        h = C.c_void_p()
        rc = lib().ductgpu_create(int(device), C.byref(h))
        if rc:
            raise DuctGPUError(rc, "ductgpu_create(device=%d) failed" % device)
        self.h = h

    def close(self):
        if self.h:
            lib().ductgpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def last_error(self):
        buf = C.create_string_buffer(512)
        lib().ductgpu_last_error(self.h, buf, 512)
        return buf.value.decode()

    def _check(self, rc):
        if rc:
            raise DuctGPUError(rc, self.last_error())
        return rc

    def synchronize(self):
        self._check(lib().ductgpu_synchronize(self.h))

    def pseudomat(self, my, mz=None):
        self._check(lib().ductgpu_pseudomat(self.h, int(my), int(mz if mz is not None else my)))
        self._my = int(my)

    def pseudomat_ex(self, my, flags=SETUP_NO_EIGEN):
        """Grid-only set-up (flags SETUP_NO_EIGEN): the eigen-decompositions
        are imported afterwards with set_operators('d'/'n')."""
        self._check(lib().ductgpu_pseudomat_ex(self.h, int(my), int(my), int(flags)))
        self._my = int(my)

    def set_gauge_point(self, iofzero):
        """The kx=0 Neumann gauge point U(iofzero+1, iofzero+1) (1-based
        interior index; 0 restores the operators' own iofzero)."""
        self._check(lib().ductgpu_set_gauge_point(self.h, int(iofzero)))

    def folded(self, bound):
        out = C.c_int()
        self._check(lib().ductgpu_get_fold(self.h, bound.encode(), C.byref(out)))
        return bool(out.value)

    def get_operators(self, bound, n):
        E = np.empty(n)
        P = np.empty((n, n), order="F")
        Q = np.empty((n, n), order="F")
        io = C.c_int()
        self._check(lib().ductgpu_get_operators(self.h, bound.encode(), _ptr(E), _ptr(P), _ptr(Q), C.byref(io)))
        return E, P, Q, io.value

    def set_operators(self, bound, E, P, PM1, iofzero=0):
        E = np.ascontiguousarray(E, dtype=np.float64)
        P = np.asfortranarray(P, dtype=np.float64)
        PM1 = np.asfortranarray(PM1, dtype=np.float64)
        self._check(lib().ductgpu_set_operators(self.h, bound.encode(), _ptr(E), _ptr(P), _ptr(PM1), int(iofzero)))

    def set_pass_kernel(self, kernel, size_class=-1):
        self._check(lib().ductgpu_set_pass_kernel(self.h, int(size_class), int(kernel)))

    def autotune(self, fields, reps=5):
        """Pick the fastest pass kernel for these fields' size class; returns it."""
        arr, keep = self._field_array(fields, False)
        out = C.c_int()
        self._check(lib().ductgpu_autotune(self.h, arr, len(fields), int(reps), C.byref(out)))
        return out.value

    def apply_tuning(self, my, mz=None, path=None):
        """The offline tuning table's settings for this grid (duct_b200/tune.py):
        pass kernel of the size class, folded or full rectangular passes.
        Returns the table entry, or None (library defaults kept)."""
        from duct_b200 import tune
        return tune.apply(self, int(my), int(mz if mz is not None else my), path or tune.TABLE)

    def set_line_kernel(self, kernel):
        """1 (default), 2: derivative lines on the FP64 tensor cores with 8 or
        16 lines per CTA, 0: the FFT kernel."""
        self._check(lib().ductgpu_set_line_kernel(self.h, int(kernel)))

    def set_rect_fold(self, on):
        """Rectangular solves: 1 (True) the flip-symmetric half blocks, the
        fields' groups of equal half-block sizes on concurrent streams; 2 the
        same in one persistent launch per solve; 0 (False) the full
        operators."""
        self._check(lib().ductgpu_set_rect_fold(self.h, int(on)))

    def set_refinement(self, steps):
        self._check(lib().ductgpu_set_refinement(self.h, int(steps)))

    def set_gauge(self, gauge):
        self._check(lib().ductgpu_set_gauge(self.h, int(gauge)))

    def helm3d(self, rhs, bound, alambda, xalp, ib=0, ipro=1, precision=PREC_FP64):
        """helm3d drop-in on host arrays: rhs (my,mz,nmodes) complex128,
        Fortran order, modified in place like the reference (walls zeroed
        for 'd').  Returns the solution."""
        assert rhs.dtype == np.complex128 and rhs.flags.f_contiguous
        my, mz, nm = rhs.shape
        sol = np.zeros_like(rhs, order="F")
        xalp = np.ascontiguousarray(xalp, dtype=np.float64)
        assert xalp.shape == (nm,)
        self._check(lib().ductgpu_helm3d(self.h, _ptr(rhs), _ptr(sol), int(ipro), bound.encode(),
                                         float(alambda), my, mz, int(ib), int(ib) + nm - 1,
                                         _ptr(xalp), int(precision)))
        return sol

    def helm3d_adjoint(self, gsol, bound, alambda, xalp, ib=0):
        """Transpose of the helm3d map applied to the cotangent gsol (host,
        complex (my,mz,nmodes)); returns grhs."""
        gsol = np.asfortranarray(gsol, dtype=np.complex128)
        my, mz, nm = gsol.shape
        out = np.zeros_like(gsol, order="F")
        xalp = np.ascontiguousarray(xalp, dtype=np.float64)
        self._check(lib().ductgpu_helm3d_adjoint(self.h, _ptr(gsol), _ptr(out), bound.encode(), float(alambda),
                                                 my, mz, int(ib), int(ib) + nm - 1, _ptr(xalp)))
        return out

    def solve_adjoint_fields_dev(self, fields):
        arr, keep = self._field_array(fields, False)
        self._check(lib().ductgpu_solve_adjoint_fields_dev(self.h, arr, len(fields)))
        return keep

    def pseudopois(self, my):
        self._check(lib().ductgpu_pseudopois(self.h, int(my)))

    def solvepois(self, U, xlambda):
        """solvepois on a real (my,my) plane; returns the solution."""
        U = np.array(U, dtype=np.float64, order="F")
        self._check(lib().ductgpu_solvepois(self.h, _ptr(U), float(xlambda), U.shape[0]))
        return U

    def solve_pois_fields_dev(self, fields):
        arr, keep = self._field_array(fields, False)
        self._check(lib().ductgpu_solve_pois_fields_dev(self.h, arr, len(fields)))
        return keep

    def preshen(self, my, bound):
        self._check(lib().ductgpu_preshen(self.h, int(my), bound.encode()))

    def helm3d_shen(self, rhs, bound, alambda, xalp, ib=0, ipro=1):
        """helm3d_shen drop-in on host arrays: rhs (my,my,nmodes) complex128,
        Fortran order, overwritten with its Chebyshev coefficients like the
        reference.  Returns the solution."""
        assert rhs.dtype == np.complex128 and rhs.flags.f_contiguous
        my, mz, nm = rhs.shape
        sol = np.zeros_like(rhs, order="F")
        xalp = np.ascontiguousarray(xalp, dtype=np.float64)
        assert xalp.shape == (nm,)
        self._check(lib().ductgpu_helm3d_shen(self.h, _ptr(rhs), _ptr(sol), int(ipro), bound.encode(),
                                              float(alambda), my, mz, int(ib), int(ib) + nm - 1, _ptr(xalp)))
        return sol

    def solve_shen_fields_dev(self, fields):
        """Like solve_fields_dev for the Shen solver (rhs overwritten)."""
        arr, keep = self._field_array(fields, False)
        self._check(lib().ductgpu_solve_shen_fields_dev(self.h, arr, len(fields)))
        return keep

    def precomp_mass_flow(self, dtp, alphak, fnu, aspect=1.0):
        """precomp_mass_flow; returns (premassfu (my,my,mrk), premassf)."""
        alphak = np.ascontiguousarray(alphak, dtype=np.float64)
        mrk = alphak.shape[0]
        m = self._my
        pf = np.zeros(mrk)
        pu = np.zeros((m, m, mrk), order="F")
        self._check(lib().ductgpu_precomp_mass_flow(self.h, float(dtp), _ptr(alphak), mrk, float(fnu),
                                                    float(aspect), _ptr(pf), _ptr(pu)))
        return pu, pf

    def impose_mass_flow(self, u, csum, krk, iflag):
        """impose_mass_flow on a host complex (my,my,...) field, modified in
        place for iflag 1; returns csum (the measured flow for iflag 0)."""
        assert u.dtype == np.complex128 and u.flags.f_contiguous
        cs = C.c_double(float(csum))
        self._check(lib().ductgpu_impose_mass_flow(self.h, C.byref(cs), int(krk), _ptr(u), int(iflag)))
        return cs.value

    def impose_mass_flow_dev(self, u, csum, krk, iflag):
        cs = C.c_double(float(csum))
        self._check(lib().ductgpu_impose_mass_flow_dev(self.h, C.byref(cs), int(krk), C.c_void_p(u.ptr),
                                                       int(iflag)))
        return cs.value

    def helm3d_batch(self, rhss, bounds, alambdas, xalp, ib=0, precision=PREC_FP64):
        """Several helm3d fields on host arrays in one pipelined call; the
        rhs arrays are modified in place like helm3d's.  Returns the sols."""
        sols = [np.zeros_like(r, order="F") for r in rhss]
        for r in rhss:
            assert r.dtype == np.complex128 and r.flags.f_contiguous and r.shape == rhss[0].shape
        my, mz, nm = rhss[0].shape
        n = len(rhss)
        pr = (C.c_void_p * n)(*[r.ctypes.data for r in rhss])
        ps = (C.c_void_p * n)(*[s_.ctypes.data for s_ in sols])
        lam = np.ascontiguousarray(alambdas, dtype=np.float64)
        xalp = np.ascontiguousarray(xalp, dtype=np.float64)
        self._check(lib().ductgpu_helm3d_batch(self.h, n, C.cast(pr, C.c_void_p), C.cast(ps, C.c_void_p),
                                               "".join(bounds).encode(), _ptr(lam), my, mz, int(ib),
                                               int(ib) + nm - 1, _ptr(xalp), int(precision)))
        return sols

    def pseudomat_temp(self, slot, my, mz, sy=1.0, sz=1.0, by=("d", "d"), bz=("d", "d")):
        self._check(lib().ductgpu_pseudomat_temp(self.h, int(slot), int(my), int(mz), float(sy), float(sz),
                                                 by[0].encode(), by[1].encode(), bz[0].encode(), bz[1].encode()))

    def helm3d_temp(self, rhs, alambda, xalp, a=1.0, b=1.0, ib=0, bcy=None, bcz=None,
                    by=("d", "d"), bz=("d", "d"), ipro=1):
        """helm3d_temp drop-in on host arrays (operator slot 0)."""
        assert rhs.dtype == np.complex128 and rhs.flags.f_contiguous
        my, mz, nm = rhs.shape
        sol = np.zeros_like(rhs, order="F")
        xalp = np.ascontiguousarray(xalp, dtype=np.float64)
        by_ = None if bcy is None else np.asfortranarray(bcy, dtype=np.float64)
        bz_ = None if bcz is None else np.asfortranarray(bcz, dtype=np.float64)
        self._check(lib().ductgpu_helm3d_temp(self.h, _ptr(rhs), _ptr(sol), int(ipro), float(a), float(b),
                                              float(alambda), my, mz, int(ib), int(ib) + nm - 1, _ptr(xalp),
                                              _ptr(by_), _ptr(bz_), by[0].encode(), by[1].encode(),
                                              bz[0].encode(), bz[1].encode()))
        return sol

    def solve_rect_fields_dev(self, fields):
        """fields: dicts(rhs, sol DeviceArray, xalp ndarray, alambda, ib, slot,
        bcy/bcz DeviceArray or None)."""
        arr = (RectField * len(fields))()
        keep = []
        for i, f in enumerate(fields):
            xalp = np.ascontiguousarray(f["xalp"], dtype=np.float64)
            keep.append(xalp)
            arr[i].rhs = f["rhs"].ptr
            arr[i].sol = f["sol"].ptr
            arr[i].xalp = xalp.ctypes.data
            arr[i].bcy = f["bcy"].ptr if f.get("bcy") is not None else None
            arr[i].bcz = f["bcz"].ptr if f.get("bcz") is not None else None
            arr[i].alambda = float(f["alambda"])
            arr[i].ib = int(f.get("ib", 0))
            arr[i].nmodes = int(xalp.shape[0])
            arr[i].slot = int(f.get("slot", 0))
        self._check(lib().ductgpu_solve_rect_fields_dev(self.h, arr, len(fields)))
        return keep

    def _field_array(self, fields, rect):
        keep = []
        if rect:
            arr = (RectField * len(fields))()
        else:
            arr = (Field * len(fields))()
        for i, f in enumerate(fields):
            xalp = np.ascontiguousarray(f["xalp"], dtype=np.float64)
            keep.append(xalp)
            arr[i].rhs = f["rhs"].ptr
            arr[i].sol = f["sol"].ptr
            arr[i].xalp = xalp.ctypes.data
            arr[i].alambda = float(f["alambda"])
            arr[i].ib = int(f.get("ib", 0))
            arr[i].nmodes = int(xalp.shape[0])
            if rect:
                arr[i].bcy = f["bcy"].ptr if f.get("bcy") is not None else None
                arr[i].bcz = f["bcz"].ptr if f.get("bcz") is not None else None
                arr[i].slot = int(f.get("slot", 0))
            else:
                arr[i].bound = f["bound"].encode()
        return arr, keep

    def graph_create(self, fields, rect=False, precision=PREC_FP64, shen=False):
        """Capture one batched solve as a CUDA graph (kind 1: rectangular,
        2: Shen, else the square diagonalisation solve); returns its id."""
        arr, keep = self._field_array(fields, rect)
        gid = C.c_int()
        kind = 1 if rect else (2 if shen else 0)
        self._check(lib().ductgpu_graph_create(self.h, kind, C.cast(arr, C.c_void_p), len(fields),
                                               int(precision), C.byref(gid)))
        return gid.value

    def graph_launch(self, gid):
        self._check(lib().ductgpu_graph_launch(self.h, int(gid)))

    def graph_destroy(self, gid):
        self._check(lib().ductgpu_graph_destroy(self.h, int(gid)))

    def solve_fields_dev(self, fields, precision=PREC_FP64):
        """fields: list of dicts(rhs=DeviceArray, sol=DeviceArray, xalp=ndarray,
        alambda=float, ib=int, bound='d'|'n')."""
        arr = (Field * len(fields))()
        keep = []
        for i, f in enumerate(fields):
            xalp = np.ascontiguousarray(f["xalp"], dtype=np.float64)
            keep.append(xalp)
            arr[i].rhs = f["rhs"].ptr if isinstance(f["rhs"], DeviceArray) else f["rhs"]
            arr[i].sol = f["sol"].ptr if isinstance(f["sol"], DeviceArray) else f["sol"]
            arr[i].xalp = xalp.ctypes.data
            arr[i].alambda = float(f["alambda"])
            arr[i].ib = int(f.get("ib", 0))
            arr[i].nmodes = int(xalp.shape[0])
            arr[i].bound = f["bound"].encode()
        self._check(lib().ductgpu_solve_fields_dev(self.h, arr, len(fields), int(precision)))
        return keep

    def transyz(self, f, cdir, iopt):
        """transyz on a host complex (my,mz,nmodes) field; returns a copy."""
        f = np.array(f, dtype=np.complex128, order="F")
        my, mz, nm = f.shape
        self._check(lib().ductgpu_transyz(self.h, _ptr(f), my, mz, nm, cdir.encode(), int(iopt)))
        return f

    def derivyz(self, u, cdir, ider, scal=1.0, what="n", du=None, aspect=1.0):
        u = np.asfortranarray(u, dtype=np.complex128)
        my, mz, nm = u.shape
        du = np.zeros_like(u, order="F") if du is None else np.array(du, dtype=np.complex128, order="F")
        self._check(lib().ductgpu_derivyz(self.h, _ptr(u), _ptr(du), my, mz, nm, cdir.encode(), int(ider),
                                          float(scal), what.encode(), float(aspect)))
        return du

    def device_array(self, shape, dtype=np.complex128):
        return DeviceArray(self, shape, dtype)

    def event_record(self, slot):
        self._check(lib().ductgpu_event_record(self.h, int(slot)))

    def event_elapsed(self, s0, s1):
        ms = C.c_float()
        self._check(lib().ductgpu_event_elapsed(self.h, int(s0), int(s1), C.byref(ms)))
        return ms.value

    def launch_count(self):
        return int(lib().ductgpu_launch_count(self.h))

    # ---- DNS operators on device fields (DeviceArray or int addresses) ----
    def derivx_dev(self, u, du, xalp, ider, scal=1.0, what="n"):
        my, mz, nm = u.shape
        self._check(lib().ductgpu_derivx_dev(self.h, _dp(u), _dp(du), my, mz, nm, _ptr(np.ascontiguousarray(
            xalp, dtype=np.float64)), int(ider), float(scal), what.encode()))

    def laplacian3d_dev(self, u, flap, xalp, scal, what="n", aspect=1.0):
        my, mz, nm = u.shape
        self._check(lib().ductgpu_laplacian3d_dev(self.h, _dp(u), _dp(flap), my, mz, nm, _ptr(np.ascontiguousarray(
            xalp, dtype=np.float64)), float(aspect), float(scal), what.encode()))

    def grad3d_dev(self, u, dxu, dyu, dzu, xalp, scal, what="n", aspect=1.0):
        my, mz, nm = u.shape
        self._check(lib().ductgpu_grad3d_dev(self.h, _dp(u), _dp(dxu), _dp(dyu), _dp(dzu), my, mz, nm,
                                             _ptr(np.ascontiguousarray(xalp, dtype=np.float64)), float(aspect),
                                             float(scal), what.encode()))

    def div3d_dev(self, u, v, w, div, xalp, scal, aspect=1.0):
        my, mz, nm = u.shape
        self._check(lib().ductgpu_div3d_dev(self.h, _dp(u), _dp(v), _dp(w), _dp(div), my, mz, nm,
                                            _ptr(np.ascontiguousarray(xalp, dtype=np.float64)), float(aspect),
                                            float(scal)))

    def update_uvwp_dev(self, u, v, w, p, phi, xalp, akk, bkk, dt, fnu, aspect=1.0):
        my, mz, nm = u.shape
        self._check(lib().ductgpu_update_uvwp_dev(self.h, _dp(u), _dp(v), _dp(w), _dp(p), _dp(phi), my, mz, nm,
                                                  _ptr(np.ascontiguousarray(xalp, dtype=np.float64)),
                                                  float(aspect), float(akk), float(bkk), float(dt), float(fnu)))

    def advection3d_dev(self, u, v, w, adv1, adv2, adv3, work, mgalx, xalp, aspect=1.0, stats2=None):
        my, mz, nm = u.shape
        self._check(lib().ductgpu_advection3d_dev(self.h, _dp(u), _dp(v), _dp(w), _dp(adv1), _dp(adv2), _dp(adv3),
                                                  _dp(work), my, mz, nm, int(mgalx),
                                                  _ptr(np.ascontiguousarray(xalp, dtype=np.float64)),
                                                  float(aspect), None if stats2 is None else _dp(stats2)))

    def vorticity_dev(self, u, v, w, vort, xalp, iflag, aspect=1.0):
        my, mz, nm = u.shape
        self._check(lib().ductgpu_vorticity_dev(self.h, _dp(u), _dp(v), _dp(w), _dp(vort), my, mz, nm,
                                                _ptr(np.ascontiguousarray(xalp, dtype=np.float64)), float(aspect),
                                                int(iflag)))

    def max_3din_dev(self, u):
        my, mz, nm = u.shape
        out = C.c_double()
        self._check(lib().ductgpu_max_3din_dev(self.h, _dp(u), my, mz, nm, C.byref(out)))
        return out.value

    def wallstressx_dev(self, u, aspect=1.0):
        my, mz = u.shape[:2]
        out = np.zeros(4)
        self._check(lib().ductgpu_wallstressx_dev(self.h, _dp(u), my, mz, float(aspect), _ptr(out)))
        return out

    def energy_fou_dev(self, u, aspect=1.0):
        my, mz, nm = u.shape
        e, e2 = C.c_double(), C.c_double()
        self._check(lib().ductgpu_energy_fou_dev(self.h, _dp(u), my, mz, nm, float(aspect), C.byref(e), C.byref(e2)))
        return e.value, e2.value

    def statistics_fou_dev(self, u, v, w, p, mean, ppb, spec):
        my, mz, nm = u.shape
        self._check(lib().ductgpu_statistics_fou_dev(self.h, _dp(u), _dp(v), _dp(w), _dp(p), my, mz, nm,
                                                     _dp(mean), _dp(ppb), _dp(spec)))

    def save_4fields_fou_hdf5_dev(self, filename, u, v, w, p, header):
        """save_4fields_fou_hdf5 of device complex (my, mz, mx1+1) fields;
        header: a dict of ductgpu_h5_header fields (sizes and scalars)."""
        h = H5Header.from_dict(header)
        self._check(lib().ductgpu_save_4fields_fou_hdf5_dev(self.h, os.fsencode(filename), _dp(u), _dp(v), _dp(w),
                                                            _dp(p), C.byref(h)))

    def read_hdf5_header(self, filename):
        h = H5Header()
        self._check(lib().ductgpu_read_hdf5_header(self.h, os.fsencode(filename), C.byref(h)))
        return h.as_dict()

    def read_4fields_fou_hdf5_dev(self, filename, u, v, w, p):
        """read_4fields_fou_hdf5 into device complex (my, mz, nmodes) fields
        (the shape of u); returns the file's header as a dict."""
        my, mz, nm = u.shape
        h = H5Header()
        self._check(lib().ductgpu_read_4fields_fou_hdf5_dev(self.h, os.fsencode(filename), _dp(u), _dp(v), _dp(w),
                                                            _dp(p), my, mz, nm, C.byref(h)))
        return h.as_dict()

    def profile(self, on=True):
        self._check(lib().ductgpu_profile_enable(self.h, int(bool(on))))

    def profile_reset(self):
        self._check(lib().ductgpu_profile_reset(self.h))

    def profile_read(self, kind):
        ms, n = C.c_double(), C.c_longlong()
        self._check(lib().ductgpu_profile_read(self.h, int(kind), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def profile_bytes(self, kind):
        b = C.c_double()
        self._check(lib().ductgpu_profile_bytes(self.h, int(kind), C.byref(b)))
        return b.value

    def profile_flops(self, kind):
        f = C.c_double()
        self._check(lib().ductgpu_profile_flops(self.h, int(kind), C.byref(f)))
        return f.value


def _dp(a):
    """Device pointer of a DeviceArray (or an int address)."""
    return C.c_void_p(a.ptr if isinstance(a, DeviceArray) else int(a))


class Dns:
    """Device-resident RK3/CN DNS of a square duct (ductgpu_dns_*): the
    substep of src/main1.f90:384-723 with the context's solver.  Fields are
    x-cut complex (my, my, M) with M = mgalx/3 modes (the 2/3 rule)."""

    def __init__(self, ctx, mgalx, alp, fnu, dt, aspect=1.0, cmassflow=True, dpdx=0.0,
                 precision=PREC_FP64, hist_cap=256):
        self.ctx = ctx
        h = C.c_void_p()
        ctx._check(lib().ductgpu_dns_create(ctx.h, int(mgalx), float(alp), float(fnu), float(dt), float(aspect),
                                            int(bool(cmassflow)), float(dpdx), int(precision), int(hist_cap),
                                            C.byref(h)))
        self.h = h
        self.my = ctx._my
        self.dt = float(dt)
        self.M = (2 * (int(mgalx) // 3)) // 2
        self.hist_cap = int(hist_cap)

    def close(self):
        if self.h:
            lib().ductgpu_dns_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_fields(self, u, v, w, p):
        arrs = [np.asfortranarray(f, dtype=np.complex128) for f in (u, v, w, p)]
        self.ctx._check(lib().ductgpu_dns_set_fields(self.h, *[_ptr(a) for a in arrs]))

    def fields(self):
        out = [np.empty((self.my, self.my, self.M), dtype=np.complex128, order="F") for _ in range(4)]
        self.ctx._check(lib().ductgpu_dns_get_fields(self.h, *[_ptr(a) for a in out]))
        return out

    def field_ptr(self, which):
        p = C.c_void_p()
        self.ctx._check(lib().ductgpu_dns_field(self.h, int(which), C.byref(p)))
        return p.value

    def set_graphs(self, on):
        self.ctx._check(lib().ductgpu_dns_set_graphs(self.h, int(bool(on))))

    def save_hdf5(self, filename, time=0.0, cfl=0.0, slip=float("nan")):
        """The state as a uvwp_NNNN.h5 file (ductgpu_dns_save_hdf5); slip
        NaN writes the wall slip measured at the last step."""
        self.ctx._check(lib().ductgpu_dns_save_hdf5(self.h, os.fsencode(filename), float(time), float(cfl),
                                                    float(slip)))

    def write_statistics_hdf5(self, filename, time=0.0, timef=0.0):
        """The accumulated statistics as a statistics_NNNN.h5 file."""
        self.ctx._check(lib().ductgpu_dns_write_statistics_hdf5(self.h, os.fsencode(filename), float(time),
                                                                float(timef)))

    def load_hdf5(self, filename):
        """Restart from a uvwp_NNNN.h5 file; returns the file's time."""
        t = C.c_double()
        self.ctx._check(lib().ductgpu_dns_load_hdf5(self.h, os.fsencode(filename), C.byref(t)))
        return t.value

    def substep(self, krk, stats=False):
        self.ctx._check(lib().ductgpu_dns_substep(self.h, int(krk), int(bool(stats))))

    def steps(self, n, stats_every=0):
        self.ctx._check(lib().ductgpu_dns_steps(self.h, int(n), int(stats_every)))

    def set_forcing(self, f=None):
        """Body force (f1, f2, f3) of complex (my, my, M) arrays, or None."""
        if f is None:
            self.ctx._check(lib().ductgpu_dns_set_forcing(self.h, None, None, None))
            return
        arrs = [np.asfortranarray(x, dtype=np.complex128) for x in f]
        self.ctx._check(lib().ductgpu_dns_set_forcing(self.h, *[_ptr(a) for a in arrs]))

    def wallstress_after(self, nsteps=1):
        J = C.c_double()
        self.ctx._check(lib().ductgpu_dns_wallstress_after(self.h, int(nsteps), C.byref(J)))
        return J.value

    def grad_wallstress(self):
        """(J, dJ/df as a (3, my, my, M) complex array) through one step."""
        g = np.zeros((3, self.M, self.my, self.my), dtype=np.complex128)   # C order = 3 Fortran fields
        J = C.c_double()
        self.ctx._check(lib().ductgpu_dns_grad_wallstress(self.h, C.byref(J), g.ctypes.data_as(C.c_void_p)))
        return J.value, np.stack([np.asfortranarray(np.transpose(g[c], (2, 1, 0))) for c in range(3)])

    def cfl(self):
        """dict(cfl, slip, cfl_max) of ductgpu_dns_cfl (cfl_max is reset)."""
        c, s, m = C.c_double(), C.c_double(), C.c_double()
        self.ctx._check(lib().ductgpu_dns_cfl(self.h, C.byref(c), C.byref(s), C.byref(m)))
        return dict(cfl=c.value, slip=s.value, cfl_max=m.value)

    def ener_lines(self, time0=0.0, interval=None):
        """The reference's 'ENER:' log lines of the recorded steps (see
        ener_line), the k-th at time time0 + k * interval (interval: the
        time between recorded steps)."""
        h, o = self.statistics()["hist"], self.statistics_omg()["hist"]
        dt = self.dt if interval is None else float(interval)
        return [ener_line(time0 + k * dt, h[k], o[k]) for k in range(min(len(h), len(o)))]

    def statistics_omg(self):
        """dict(om2 (3,my,my): omx2, omy2, omz2; hist (nhist,16): sector
        energies [5] and |Re| integrals [5] of om_x, energy_fou of om_x,
        om_y, om_z, the same with mode 0) -- ductgpu_dns_statistics_omg."""
        my = self.my
        om2 = np.zeros((my, my, 3), order="F")
        hist = np.zeros((max(self.hist_cap, 1), 16))
        nh = C.c_int()
        self.ctx._check(lib().ductgpu_dns_statistics_omg(self.h, _ptr(om2), _ptr(hist), C.byref(nh)))
        return dict(om2=np.moveaxis(om2, 2, 0).copy(), hist=hist[:nh.value].copy())

    def statistics(self):
        """dict(nstat, mean (4,my,my), prod (6,my,my), ppb (my,my), spec
        (4,7,M), hist (nhist,10), divmax (3,)) -- the oracle's layout."""
        my, M = self.my, self.M
        mean = np.zeros((my, my, 4), order="F")
        prod = np.zeros((my, my, 6), order="F")
        ppb = np.zeros((my, my), order="F")
        spec = np.zeros((M, 7, 4), order="F")
        hist = np.zeros((max(self.hist_cap, 1), 10))
        ns, nh = C.c_int(), C.c_int()
        dv = np.zeros(3)
        self.ctx._check(lib().ductgpu_dns_statistics(self.h, _ptr(mean), _ptr(prod), _ptr(ppb), _ptr(spec),
                                                     _ptr(hist), C.byref(ns), C.byref(nh), _ptr(dv)))
        return dict(nstat=ns.value, mean=np.moveaxis(mean, 2, 0).copy(), prod=np.moveaxis(prod, 2, 0).copy(),
                    ppb=ppb, spec=np.transpose(spec, (2, 1, 0)).copy(), hist=hist[:nh.value].copy(), divmax=dv)


__all__ = ["Context", "Dns", "DeviceArray", "DuctGPUError", "H5Header", "lib", "LIB_PATH", "EXPORTS",
           "uvwp_filename", "statistics_filename", "read_hdf5_header", "ener_line", "fortran_e15_8",
           "PREC_FP64", "PREC_MIXED", "GAUGE_POINT", "GAUGE_MEAN"]
