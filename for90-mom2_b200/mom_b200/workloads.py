"""Synthetic workloads of the linear PMCHWT path (seeded, no datasets).

    sphere(s)          icosphere, r = 50 nm, eps = -9 + 1.3i inside, vacuum outside
    sweep_meshes()     the s=3 sphere plus three seeded triaxial ellipsoids
                       (semi-axes U(30, 70) nm, 2-3 subdivisions), default_rng(3)
    drude_eps(wl)      eps(w) = 1 - wp^2 / (w^2 + i gamma w), hbar wp = 9.0 eV,
                       hbar gamma = 0.07 eV
    sweep_wavelengths  64 vacuum wavelengths uniform on 400-900 nm
    perturbed(s)       radially perturbed sphere, real Y_lm for l <= 4,
                       c_lm ~ N(0, 0.03^2), default_rng(4)
    core_shell(s)      core r = 40 nm (eps 2.13) in a shell r = 60 nm
                       (eps -9 + 1.3i) in vacuum; 3 domains
    incidences(k)      k pw_elliptic sources, theta = arccos U(-1, 1),
                       phi = U(0, 2 pi), phase = exp(i U(0, 2 pi)), default_rng(5)

Each mesh function returns (nodes [nm], faces, face_ids, domains).
"""
from __future__ import annotations

import numpy as np

from . import meshgen

EPS_AU = -9.0 + 1.3j
EPS_SILICA = 2.13
HBAR_EVS = 6.582119569e-16  # eV s
C0_PHYS = 2.99792458e8


def sphere(s: int, radius: float = 50.0):
    nodes, faces = meshgen.icosphere(s, radius)
    return nodes, faces, np.ones(len(faces), int), [[1], [-1]]


def perturbed(s: int, radius: float = 50.0):
    nodes, faces = meshgen.perturbed_sphere(s, radius, lmax=4, sigma=0.03, seed=4)
    return nodes, faces, np.ones(len(faces), int), [[1], [-1]]


def core_shell(s: int, r_core: float = 40.0, r_shell: float = 60.0):
    n1, f1 = meshgen.icosphere(s, r_core)
    n2, f2 = meshgen.icosphere(s, r_shell)
    nodes = np.vstack([n1, n2])
    faces = np.vstack([f1, f2 + len(n1)])
    ids = np.r_[np.full(len(f1), 1), np.full(len(f2), 2)]
    return nodes, faces, ids, [[2], [-2, 1], [-1]]


def sweep_meshes():
    """[(name, mesh)] of the uneven wavelength-sweep set."""
    rng = np.random.default_rng(3)
    axes = rng.uniform(30.0, 70.0, (3, 3))
    subs = rng.integers(2, 4, 3)
    out = [("sphere s=3", sphere(3))]
    for i in range(3):
        nodes, faces = meshgen.ellipsoid(int(subs[i]), axes[i])
        out.append(("ellipsoid s=%d axes=(%.1f, %.1f, %.1f) nm" % (subs[i], *axes[i]),
                    (nodes, faces, np.ones(len(faces), int), [[1], [-1]])))
    return out


def sweep_wavelengths(n: int = 64):
    return np.linspace(400e-9, 900e-9, n)


def drude_eps(wl):
    """Drude permittivity at vacuum wavelength wl (physical omega = 2 pi c / wl)."""
    w = 2.0 * np.pi * C0_PHYS / np.asarray(wl, dtype=np.float64)
    wp = 9.0 / HBAR_EVS
    g = 0.07 / HBAR_EVS
    return 1.0 - wp * wp / (w * w + 1j * g * w)


def incidences(k: int, seed: int = 5):
    """k pw_elliptic sources as dicts for the Solver (angles in radians)."""
    from . import DEGTORAD, src_pw_elliptic
    rng = np.random.default_rng(seed)
    th = np.arccos(rng.uniform(-1.0, 1.0, k))
    ph = rng.uniform(0.0, 2.0 * np.pi, k)
    phase = np.exp(1j * rng.uniform(0.0, 2.0 * np.pi, k))
    return [src_pw_elliptic(t / DEGTORAD, p / DEGTORAD, z) for t, p, z in zip(th, ph, phase)]
