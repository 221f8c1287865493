"""Mie series for a homogeneous sphere (test infrastructure: a physics anchor).

Written from the textbook Lorenz-Mie coefficients (Bohren & Huffman,
"Absorption and Scattering of Light by Small Particles", eqs. 4.53, 4.61-4.62),
not from the reference, which ships no Mie code.  Used to sanity-check the
oracle and the GPU solver on sphere meshes.
"""
from __future__ import annotations

import numpy as np
from scipy.special import spherical_jn, spherical_yn


def mie_cross_sections(radius: float, wavelength: float, n_sphere: complex, n_medium: float = 1.0,
                       nmax: int | None = None):
    """Return (sigma_ext, sigma_sca, sigma_abs) in m^2 for a sphere of given radius (m)."""
    k = 2 * np.pi * n_medium / wavelength
    x = k * radius
    m = complex(n_sphere) / n_medium
    if nmax is None:
        nmax = int(np.ceil(x + 4.05 * x ** (1.0 / 3.0) + 2)) + 10
    n = np.arange(1, nmax + 1)
    mx = m * x

    def psi(nn, z):
        return z * spherical_jn(nn, z)

    def dpsi(nn, z):
        return spherical_jn(nn, z) + z * spherical_jn(nn, z, derivative=True)

    def xi(nn, z):
        return z * (spherical_jn(nn, z) + 1j * spherical_yn(nn, z))

    def dxi(nn, z):
        h = spherical_jn(nn, z) + 1j * spherical_yn(nn, z)
        dh = spherical_jn(nn, z, derivative=True) + 1j * spherical_yn(nn, z, derivative=True)
        return h + z * dh

    px, dpx = psi(n, x), dpsi(n, x)
    pmx, dpmx = psi(n, mx), dpsi(n, mx)
    xx, dxx = xi(n, x), dxi(n, x)
    an = (m * pmx * dpx - px * dpmx) / (m * pmx * dxx - xx * dpmx)
    bn = (pmx * dpx - m * px * dpmx) / (pmx * dxx - m * xx * dpmx)
    qext = 2.0 / x ** 2 * np.sum((2 * n + 1) * np.real(an + bn))
    qsca = 2.0 / x ** 2 * np.sum((2 * n + 1) * (np.abs(an) ** 2 + np.abs(bn) ** 2))
    g = np.pi * radius ** 2
    return qext * g, qsca * g, (qext - qsca) * g
