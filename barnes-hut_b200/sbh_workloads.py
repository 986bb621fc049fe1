"""Seeded synthetic workloads with the shapes and distributions of the
benchmark configurations (no dataset is fetched; everything is generated from
``numpy.random.default_rng(seed)``).

* ``uniform_cube``      N points uniform in [0,1)^3, masses 1/N
* ``plummer``           Plummer sphere (scale radius a, truncated at r_max = 10a),
                        equal masses, radius by the exact inverse CDF of the
                        truncated mass profile M(r) = r^3 / (r^2 + a^2)^{3/2}
* ``ellipsoid_surface`` oriented points area-uniform on a triaxial ellipsoid,
                        outward normals grad F / |grad F|, weights = area / N
* ``forest``            many independent Plummer systems with N log-uniform
* ``perturbed_lattice`` k^3 lattice in the unit box displaced by a Gaussian
                        random field with P(k) ~ k^-2 cut at the Nyquist wavenumber
"""
from __future__ import annotations

import numpy as np


def uniform_cube(n: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 3), dtype=np.float64).astype(np.float32)
    masses = np.full(n, 1.0 / n, np.float32)
    return pts, masses


def plummer(n: int, seed: int = 0, a: float = 1.0, r_max_over_a: float = 10.0):
    """Equal-mass Plummer sphere truncated at r_max, total mass 1."""
    rng = np.random.default_rng(seed)
    rmax = r_max_over_a * a
    m_max = rmax**3 / (rmax**2 + a**2) ** 1.5  # M(r_max) / M_total for a = scale
    x = rng.random(n) * m_max
    x = np.clip(x, 1e-300, None)
    r = a / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
    cth = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    sth = np.sqrt(1.0 - cth * cth)
    pts = np.stack([r * sth * np.cos(phi), r * sth * np.sin(phi), r * cth], axis=1).astype(np.float32)
    masses = np.full(n, 1.0 / n, np.float32)
    return pts, masses


def _ellipsoid_area(a: float, b: float, c: float, nq: int = 400) -> float:
    """Surface area of the ellipsoid by Gauss-Legendre quadrature in (theta, phi)."""
    xt, wt = np.polynomial.legendre.leggauss(nq)
    th = (xt + 1.0) * (np.pi / 2.0)
    wth = wt * (np.pi / 2.0)
    ph = (xt + 1.0) * np.pi
    wph = wt * np.pi
    T, P = np.meshgrid(th, ph, indexing="ij")
    st, ct, sp, cp = np.sin(T), np.cos(T), np.sin(P), np.cos(P)
    # |r_theta x r_phi| for r = (a st cp, b st sp, c ct)
    nx = b * c * st * st * cp
    ny = a * c * st * st * sp
    nz = a * b * st * ct
    dA = np.sqrt(nx * nx + ny * ny + nz * nz)
    return float(np.einsum("i,j,ij->", wth, wph, dA))


def ellipsoid_surface(n: int, seed: int = 0, axes=(1.0, 0.7, 0.5)):
    """Area-uniform oriented samples on x^2/a^2 + y^2/b^2 + z^2/c^2 = 1."""
    a, b, c = axes
    rng = np.random.default_rng(seed)
    out = np.zeros((0, 3))
    gmax = max(b * c, a * c, a * b)
    while out.shape[0] < n:
        k = int((n - out.shape[0]) * 1.6) + 1024
        v = rng.normal(size=(k, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        p = v * np.array([a, b, c])
        # area element of the map sphere -> ellipsoid is proportional to
        # |(bc x, ac y, ab z)| for the unit-sphere point (x, y, z)
        g = np.sqrt((b * c * v[:, 0]) ** 2 + (a * c * v[:, 1]) ** 2 + (a * b * v[:, 2]) ** 2)
        keep = rng.random(k) * gmax < g
        out = np.concatenate([out, p[keep]], axis=0)
    pts = out[:n]
    grad = pts / np.array([a * a, b * b, c * c])
    nrm = grad / np.linalg.norm(grad, axis=1, keepdims=True)
    area = _ellipsoid_area(a, b, c)
    w = np.full(n, area / n, np.float32)
    return pts.astype(np.float32), nrm.astype(np.float32), w


def ellipsoid_inside(q, axes=(1.0, 0.7, 0.5)):
    a, b, c = axes
    q = np.asarray(q, np.float64)
    return (q[:, 0] / a) ** 2 + (q[:, 1] / b) ** 2 + (q[:, 2] / c) ** 2 < 1.0


def torus_mesh(R: float = 1.0, r: float = 0.4, nu: int = 128, nv: int = 64):
    """Closed triangle mesh of the torus (sqrt(x^2 + y^2) - R)^2 + z^2 = r^2:
    vertices on an nu x nv grid of the angles around the z axis (u) and
    around the tube (v), two triangles per grid cell, ordered so that
    e1 x e2 points outward. Returns (V (nu*nv, 3) float32, F (2*nu*nv, 3)
    int32)."""
    u = 2 * np.pi * np.arange(nu) / nu
    v = 2 * np.pi * np.arange(nv) / nv
    U, Vv = np.meshgrid(u, v, indexing="ij")
    ring = R + r * np.cos(Vv)
    V = np.stack([ring * np.cos(U), ring * np.sin(U), r * np.sin(Vv)], axis=-1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    a = i * nv + j
    b = ((i + 1) % nu) * nv + j
    c = ((i + 1) % nu) * nv + (j + 1) % nv
    d = i * nv + (j + 1) % nv
    F = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)])
    return V.astype(np.float32), F.astype(np.int32)


def torus_inside(q, R: float = 1.0, r: float = 0.4):
    q = np.asarray(q, np.float64)
    return (np.sqrt(q[:, 0] ** 2 + q[:, 1] ** 2) - R) ** 2 + q[:, 2] ** 2 < r * r


def uniform_box_queries(m: int, seed: int = 1, half: float = 1.5):
    rng = np.random.default_rng(seed)
    return rng.uniform(-half, half, (m, 3)).astype(np.float32)


def forest(num_systems: int = 256, n_lo: int = 1000, n_hi: int = 200000, seed: int = 0):
    """Independent Plummer systems; N log-uniform in [n_lo, n_hi]. Returns a
    list of (points, masses) and the sizes."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), num_systems)).astype(np.int64)
    systems = [plummer(int(s), seed=seed * 100003 + i + 1) for i, s in enumerate(sizes)]
    return systems, sizes


def perturbed_lattice(k: int = 128, seed: int = 0, rms_cells: float = 0.2):
    """k^3 lattice in [0,1)^3 displaced by a Gaussian random field with
    P(k) ~ k^-2 for 0 < |k| <= k_Nyquist, scaled to an rms displacement of
    rms_cells lattice spacings. Returns (points, masses, displacement)."""
    rng = np.random.default_rng(seed)
    g = np.fft.fftfreq(k) * k  # integer wavenumbers
    kx, ky, kz = np.meshgrid(g, g, g, indexing="ij")
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    amp = np.zeros_like(kk)
    nz = (kk > 0) & (kk <= k / 2)
    amp[nz] = kk[nz] ** -1.0  # sqrt(P) with P ~ k^-2
    disp = np.zeros((k, k, k, 3))
    for d in range(3):
        white = rng.normal(size=(k, k, k)) + 1j * rng.normal(size=(k, k, k))
        disp[..., d] = np.real(np.fft.ifftn(white * amp))
    disp *= (rms_cells / k) / np.sqrt(np.mean(np.sum(disp * disp, axis=-1)))
    lat = (np.stack(np.meshgrid(np.arange(k), np.arange(k), np.arange(k), indexing="ij"), axis=-1) + 0.5) / k
    pts = (lat + disp).reshape(-1, 3).astype(np.float32)
    masses = np.full(pts.shape[0], 1.0 / pts.shape[0], np.float32)
    return pts, masses, disp.reshape(-1, 3).astype(np.float32)
