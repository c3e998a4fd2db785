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
