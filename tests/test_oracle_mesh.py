"""The oracle's mesh surface sampler (the restatement the GPU sampler is
checked against): splitmix64 known answers, face geometry of a closed torus
mesh, and the sampling distribution of python/old_interface/sampler.py:63-78
(area-proportional faces, uniform points inside them)."""
import numpy as np
import pytest

import sbh_oracle as O
import sbh_workloads as W


def test_splitmix64_known_answers():
    # the first outputs of splitmix64 seeded with 0
    g = np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        z = O.splitmix64_mix(np.arange(1, 4, dtype=np.uint64) * g)
    assert [int(x) for x in z] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_torus_mesh_geometry():
    R, r = 1.0, 0.4
    V, F = W.torus_mesh(R, r, 128, 64)
    area2, nrm = O.mesh_face_geometry(V, F)
    # polygonal torus area approaches 4 pi^2 R r from below
    area = 0.5 * area2.sum()
    assert 0.995 * 4 * np.pi ** 2 * R * r < area < 4 * np.pi ** 2 * R * r
    np.testing.assert_allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-6)
    # outward: the normal points away from the tube's centre circle
    cen = V[F].mean(axis=1).astype(np.float64)
    ring = cen.copy()
    ring[:, 2] = 0
    ring *= R / np.linalg.norm(ring, axis=1, keepdims=True)
    assert (np.sum((cen - ring) * nrm, axis=1) > 0).all()


def test_sampler_distribution_and_determinism():
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 2], [3, 0, 2]], np.float32)
    F = np.array([[0, 1, 2], [0, 3, 4], [1, 2, 3], [0, 0, 1]], np.int32)  # the last face is degenerate
    n = 200000
    pts, nrm, w, face = O.sample_points_on_mesh(n, V, F, seed=7)
    area2, _ = O.mesh_face_geometry(V, F)
    assert area2[3] == 0 and not (face == 3).any()
    # face counts follow the areas (chi-square, 2 degrees of freedom)
    p = area2[:3] / area2[:3].sum()
    cnt = np.bincount(face, minlength=4)[:3]
    chi2 = ((cnt - n * p) ** 2 / (n * p)).sum()
    assert chi2 < 13.8  # p = 0.001
    # every point lies in its face: barycentric coordinates from the 2 x 2
    # normal equations of p - v0 = b1 e1 + b2 e2
    v0, v1, v2 = (V[F[face, k]].astype(np.float64) for k in range(3))
    e1, e2, dp = v1 - v0, v2 - v0, pts.astype(np.float64) - v0
    g11, g12, g22 = (e1 * e1).sum(1), (e1 * e2).sum(1), (e2 * e2).sum(1)
    r1, r2 = (e1 * dp).sum(1), (e2 * dp).sum(1)
    det = g11 * g22 - g12 * g12
    b1, b2 = (g22 * r1 - g12 * r2) / det, (g11 * r2 - g12 * r1) / det
    assert (b1 > -1e-5).all() and (b2 > -1e-5).all() and (b1 + b2 < 1 + 1e-5).all()
    # and on the face's plane
    resid = dp - b1[:, None] * e1 - b2[:, None] * e2
    assert np.abs(resid).max() < 1e-5
    # uniform inside a face: the mean barycentric pair is (1/3, 1/3)
    # (standard deviation 1/sqrt(18 n) per coordinate)
    np.testing.assert_allclose([b1.mean(), b2.mean()], [1 / 3, 1 / 3], atol=5 / np.sqrt(18 * n))
    np.testing.assert_allclose(w, 0.5 * area2.sum() / n, rtol=1e-6)
    # sample i depends on (seed, i) only
    p2, _, _, f2 = O.sample_points_on_mesh(1000, V, F, seed=7)
    np.testing.assert_array_equal(p2, pts[:1000])
    np.testing.assert_array_equal(f2, face[:1000])
    p3, *_ = O.sample_points_on_mesh(1000, V, F, seed=8)
    assert not np.array_equal(p3, p2)


@pytest.mark.parametrize("nu,nv", [(64, 32)])
def test_sampled_torus_winding_number(nu, nv):
    """Winding number of samples of the closed torus mesh (FP64 direct sum):
    about 1 inside the tube and 0 outside, away from the surface."""
    V, F = W.torus_mesh(1.0, 0.4, nu, nv)
    pts, nrm, w, _ = O.sample_points_on_mesh(40000, V, F, seed=3)
    rng = np.random.default_rng(4)
    q = rng.uniform(-1.5, 1.5, (600, 3)).astype(np.float32)
    d = np.abs(np.sqrt((np.sqrt(q[:, 0] ** 2 + q[:, 1] ** 2) - 1.0) ** 2 + q[:, 2] ** 2) - 0.4)
    q = q[d > 0.1]
    wn = O.direct_winding_number(pts, nrm, w, q)
    inside = W.torus_inside(q)
    assert np.abs(wn[inside] - 1).mean() < 0.05
    assert np.abs(wn[~inside]).mean() < 0.05


def _one_face(p):
    return np.asarray(p, np.float32), np.array([[0, 1, 2]])


def test_vertex_sources_voronoi_known_answers():
    """Mixed Voronoi areas (Meyer et al. 2003) on single faces: an equilateral
    face splits evenly; a right angle takes the square up to the hypotenuse's
    midpoint (1/4 of legs 1 x 1) and the other corners 1/8; an obtuse corner
    takes half the area and the others a quarter."""
    s3 = np.sqrt(3.0)
    n, m = O.mesh_vertex_sources(*_one_face([[0, 0, 0], [1, 0, 0], [0.5, s3 / 2, 0]]))
    np.testing.assert_allclose(m, np.full(3, s3 / 12), rtol=1e-6)
    np.testing.assert_allclose(n, np.tile([0.0, 0.0, 1.0], (3, 1)), atol=1e-12)
    _, m = O.mesh_vertex_sources(*_one_face([[0, 0, 0], [1, 0, 0], [0, 1, 0]]))
    np.testing.assert_allclose(m, [0.25, 0.125, 0.125], rtol=1e-12)
    V, F = _one_face([[0, 0, 0], [1, 0.1, 0], [-1, 0.1, 0]])
    area = 0.5 * abs(np.cross(V[1].astype(np.float64) - V[0], V[2].astype(np.float64) - V[0])[2])
    _, m = O.mesh_vertex_sources(V, F)
    np.testing.assert_allclose(m, [area / 2, area / 4, area / 4], rtol=1e-12)
    # corner order does not matter: the obtuse corner moved to position 2
    _, m = O.mesh_vertex_sources(V[[1, 2, 0]], F)
    np.testing.assert_allclose(m, [area / 4, area / 4, area / 2], rtol=1e-12)


def test_vertex_sources_torus():
    """On the closed torus mesh the masses sum to the surface area (the sum
    of the face areas) and the area-weighted normals point along the
    analytic torus normal."""
    V, F = W.torus_mesh(1.0, 0.4, 64, 32)
    n, m = O.mesh_vertex_sources(V, F)
    area2, _ = O.mesh_face_geometry(V, F)
    np.testing.assert_allclose(m.sum(), 0.5 * area2.sum(), rtol=1e-12)
    assert (m > 0).all()
    np.testing.assert_allclose(np.linalg.norm(n, axis=1), 1.0, rtol=1e-12)
    p = V.astype(np.float64)
    rho = np.hypot(p[:, 0], p[:, 1])
    c = np.stack([p[:, 0] / rho, p[:, 1] / rho, np.zeros_like(rho)], axis=1)  # ring centre direction
    radial = p - c * 1.0
    radial /= np.linalg.norm(radial, axis=1, keepdims=True)
    assert np.einsum("ij,ij->i", n, radial).min() > 0.99


def test_vertex_sources_degenerate_and_unused():
    """A zero-area face adds nothing; a vertex without faces keeps mass 0 and
    a zero normal."""
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [2, 0, 0], [5, 5, 5]], np.float32)
    F = np.array([[0, 1, 2], [0, 1, 3]])  # the second face is collinear
    n, m = O.mesh_vertex_sources(V, F)
    np.testing.assert_allclose(m, [0.25, 0.125, 0.125, 0.0, 0.0], rtol=1e-12)
    assert np.all(n[3:] == 0.0)
