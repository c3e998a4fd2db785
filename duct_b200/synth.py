"""Seeded synthetic inputs of the benchmark configurations.

The reference ships no input data (no restart fields, no logs), so every
right-hand side is generated here from a documented generator that any
implementation can reproduce:

* splitmix64 stream (Steele, Lea & Flood 2014) started at ``seed``; uniform
  doubles are the top 53 bits; normals come from Box-Muller pairs
  (Re from the cosine branch, Im from the sine branch);
* complex Chebyshev coefficients c(i, j, k) ~ N(0,1) + i N(0,1) drawn in
  column-major order of (y-index i, z-index j, mode k), scaled by
  1/((1+i)(1+j))^2;
* mapped to collocation values with the reference's inverse Chebyshev
  transform in y then z (src/tchebw.f:119-134):
  u(p, q) = sum_ij c(i, j) cos(pi p i/(my-1)) cos(pi q j/(mz-1));
* the imaginary part of Fourier mode 0 is zero (src/int2d3d.f90:43).
"""
import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed, count):
    """``count`` successive splitmix64 outputs as uint64."""
    with np.errstate(over="ignore"):
        i = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def normals_complex(seed, count):
    """``count`` complex N(0,1)+iN(0,1) values (Box-Muller on splitmix64)."""
    z = splitmix64(seed, 2 * count)
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log1p(-u1))
    th = 2.0 * np.pi * u2
    return r * np.cos(th) + 1j * (r * np.sin(th))


def cheb_to_phys_matrix(m):
    """T[p, i] = cos(pi p i/(m-1)): the inverse transform of src/tchebw.f."""
    p = np.arange(m)
    return np.cos(np.pi * np.outer(p, p) / (m - 1))


def chebyshev_rhs(my, mz, nmodes, seed=0, ib=0):
    """Complex (my, mz, nmodes) Fortran-ordered RHS in physical space."""
    c = normals_complex(seed, my * mz * nmodes).reshape((my, mz, nmodes), order="F")
    i = np.arange(my)[:, None, None]
    j = np.arange(mz)[None, :, None]
    c = c / ((1.0 + i) * (1.0 + j)) ** 2
    Ty, Tz = cheb_to_phys_matrix(my), cheb_to_phys_matrix(mz)
    f = np.einsum("pi,ijk,qj->pqk", Ty, c, Tz, optimize=True)
    f = np.asfortranarray(f)
    if ib == 0:
        f[:, :, 0] = f[:, :, 0].real
    return f


def config(name):
    """Workloads of the benchmark configurations (square collocation grid)."""
    if name == "cfg0":
        nu, dt = 1.0 / 2000.0, 1.0e-3
        return dict(my=33, mz=33, nmodes=17, alp=1.0, fields=[("u", "d", 2.0 / (nu * dt))])
    if name == "cfg1":
        nu, dt = 1.0 / 2000.0, 1.0e-3
        h = 2.0 / (nu * dt)
        return dict(my=129, mz=129, nmodes=64, alp=0.5,
                    fields=[("u", "d", h), ("v", "d", h), ("w", "d", h), ("p", "n", 0.0)])
    raise KeyError(name)


def cgl_derivative(m, s=1.0):
    """Nodes x_j = -s cos(pi j/(m-1)) and the collocation first-derivative
    matrix on them (CHQZ eq. 2.4.31, the matrix of src/pseudomat.f90:83-107)."""
    n = m - 1
    j = np.arange(m)
    x = -np.cos(np.pi * j / n)
    c = np.where((j == 0) | (j == n), 2.0, 1.0)
    X = x[:, None] - x[None, :]
    sgn = np.where((j[:, None] + j[None, :]) % 2 == 0, 1.0, -1.0)
    D = np.zeros((m, m))
    off = ~np.eye(m, dtype=bool)
    D[off] = (c[:, None] / c[None, :] * sgn / np.where(off, X, 1.0))[off]
    D[j, j] = -0.5 * x / np.where((j == 0) | (j == n), 1.0, 1.0 - x * x)
    D[0, 0] = -(2.0 * n * n + 1.0) / 6.0
    D[n, n] = (2.0 * n * n + 1.0) / 6.0
    return s * x, D / s


def laminar_profile(m, aspect=1.0):
    """The laminar square-duct profile U(y, z) (my = mz = m) with max U = 1:
    U = W / max W where lap W = -1, W = 0 on the walls (the problem the
    reference tabulates in get_dpdx, src/operators.F:2496-2507).  Returns
    (U, dpval) with lap U = -dpval."""
    x, D = cgl_derivative(m)
    D2 = D @ D
    B = D2[1:-1, 1:-1]
    E, P = np.linalg.eig(B)
    E, P = E.real, P.real
    Q = np.linalg.inv(P)
    F = -np.ones((m - 2, m - 2))
    W = np.zeros((m, m))
    W[1:-1, 1:-1] = P @ ((Q @ F @ Q.T) / (E[:, None] + E[None, :])) @ P.T
    mx = W.max()
    return W / mx, 1.0 / mx


def dns_initial(mgalx, m, alp, amp, seed=0, kmax=8, nterms=4):
    """Seeded initial state of a square-duct DNS: x-cut complex
    (m, m, M) fields u, v, w, p with M = mgalx/3 (the 2/3 rule: mx =
    2 (mgalx/3), M = mx/2 modes, src/mod.f90:86-91).  u mode 0 is the
    laminar profile (max 1); the perturbation is the curl of a vector
    potential psi = (1-y^2)^2 (1-z^2)^2 phi, phi a seeded random combination
    of T_a(y) T_b(z) (a, b < nterms) in Fourier modes 0..kmax, so it is
    divergence-free for the collocation derivatives and zero on the walls;
    it is scaled to max |u'| = amp (over the physical grid).  p = 0.
    Returns (u, v, w, p, dpval)."""
    mx = 2 * (mgalx // 3)
    M = mx // 2
    x, D = cgl_derivative(m)
    U, dpval = laminar_profile(m)
    T = np.cos(np.arange(nterms)[None, :] * np.arccos(np.clip(x, -1.0, 1.0))[:, None])   # T_a(x_j)
    bub = (1.0 - x * x) ** 2
    kk = min(kmax, M - 1)
    r = normals_complex(seed, 3 * nterms * nterms * (kk + 1)).reshape((3, kk + 1, nterms, nterms))
    r[:, 0] = r[:, 0].real
    psi = np.einsum("ja,ckab,lb->cjlk", T, r, T) * (bub[:, None] * bub[None, :])[None, :, :, None]
    kx = alp * np.arange(kk + 1)
    Dy = lambda f: np.einsum("ij,jlk->ilk", D, f)
    Dz = lambda f: np.einsum("lj,ijk->ilk", D, f)
    px, py, pz = psi
    up = Dy(pz) - Dz(py)
    vp = Dz(px) - 1j * kx * pz
    wp = 1j * kx * py - Dy(px)
    # physical maximum of the perturbation (inverse real FFT along x)
    def phys(f):
        g = np.zeros((m, m, mgalx // 2 + 1), dtype=np.complex128)
        g[:, :, :kk + 1] = f
        return np.fft.irfft(g, n=mgalx, axis=2) * mgalx
    mag = np.sqrt(phys(up) ** 2 + phys(vp) ** 2 + phys(wp) ** 2).max()
    s = amp / mag
    u = np.zeros((m, m, M), dtype=np.complex128, order="F")
    v, w, p = (np.zeros_like(u, order="F") for _ in range(3))
    u[:, :, 0] = U
    u[:, :, :kk + 1] += s * up
    v[:, :, :kk + 1] = s * vp
    w[:, :, :kk + 1] = s * wp
    for f in (u, v, w):
        f[:, :, 0] = f[:, :, 0].real
        f[0, :, :] = f[-1, :, :] = f[:, 0, :] = f[:, -1, :] = 0.0
    return u, v, w, p, dpval


def dns_config(name):
    """The DNS configurations: cfg3 (adjoint check: mgalx = 64, my = mz = 65,
    Lx = 2 pi, Re_b = 2000, one RK3/CN step, 5 % perturbation) and cfg4
    (mgalx = 256, my = mz = 193, Lx = 4 pi, Re_b = 4400, dt = 2e-4, 200
    steps, 10 % perturbation).  The bulk Reynolds number is the reference's
    Re = Q / (4 nu) with Q the flow rate (src/operators.F:2335); Q is that of
    the laminar profile with max 1 (the initial mean flow), and the flow rate
    is held by impose_mass_flow (CMASSFLOW).  cfg3's dt is not given and is
    taken as 1e-3."""
    if name == "cfg3":
        return dict(mgalx=64, my=65, alp=1.0, re_b=2000.0, dt=1.0e-3, steps=1, amp=0.05)
    if name == "cfg4":
        return dict(mgalx=256, my=193, alp=0.5, re_b=4400.0, dt=2.0e-4, steps=200, amp=0.10)
    raise KeyError(name)
