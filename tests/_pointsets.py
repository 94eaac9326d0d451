"""Seeded synthetic point sets with the shapes and distributions of the
benchmark workloads (shared by tests and bench)."""
from __future__ import annotations

import numpy as np


def uniform_cube(n, seed):
    return np.random.default_rng(seed).random((3, n))


def sphere_plummer(n, seed, plummer_scale=0.1):
    """Half on the unit sphere surface (g/|g|, g ~ N(0, I3)), half Plummer
    with scale ``plummer_scale`` (r = a / sqrt(u^(-2/3) - 1), isotropic)."""
    rng = np.random.default_rng(seed)
    n1 = n // 2
    g = rng.standard_normal((3, n1))
    sph = g / np.linalg.norm(g, axis=0)
    n2 = n - n1
    u = rng.uniform(1e-12, 1.0, n2)
    r = plummer_scale / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    # cap the heavy tail so the tree's root box stays finite and modest
    r = np.minimum(r, 10.0)
    d = rng.standard_normal((3, n2))
    d /= np.linalg.norm(d, axis=0)
    return np.concatenate([sph, r * d], axis=1)


def sphere_quadrature(ntheta):
    """Nodes and weights of a tensor quadrature on the unit sphere:
    Gauss-Legendre in cos(theta) (ntheta nodes) times the midpoint rule in
    phi (2 ntheta nodes); exact for spherical harmonics of degree < 2 ntheta.
    Returns (points (3, n), weights (n,)); the points are also the normals."""
    x, w = np.polynomial.legendre.leggauss(ntheta)
    nphi = 2 * ntheta
    phi = (np.arange(nphi) + 0.5) * 2.0 * np.pi / nphi
    ct = np.repeat(x, nphi)
    st = np.sqrt(1.0 - ct * ct)
    ph = np.tile(phi, ntheta)
    pts = np.stack([st * np.cos(ph), st * np.sin(ph), ct])
    return pts, np.repeat(w, nphi) * (2.0 * np.pi / nphi)
