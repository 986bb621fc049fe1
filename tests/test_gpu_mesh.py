"""GPU mesh surface sampler (sbh_sample_mesh_surface) against the oracle's
restatement (oracle/sbh_oracle.py sample_points_on_mesh): the same samples
bit for bit, and the winding number of a sampled closed mesh through the
native tree."""
import numpy as np
import pytest
import torch

import sbh_b200 as B
import sbh_oracle as O
import sbh_workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nu,nv,n,seed", [(32, 16, 100000, 0), (128, 64, 262144, 12345), (3, 3, 1000, 2**63 + 5)])
def test_mesh_sampler_matches_oracle(cuda, nu, nv, n, seed):
    V, F = W.torus_mesh(1.0, 0.4, nu, nv)
    pts, nrm, w = B.sample_points_on_mesh(n, V, F, seed=seed)
    want_p, want_n, want_w, _ = O.sample_points_on_mesh(n, V, F, seed=seed)
    pts, nrm, w = pts.cpu().numpy(), nrm.cpu().numpy(), w.cpu().numpy()
    # the cumulative areas are summed in another order on the device: a sample
    # may pick the neighbouring face only when its target lands within a few
    # ulps of a face boundary
    diff = np.any(pts != want_p, axis=1) | np.any(nrm != want_n, axis=1)
    assert diff.sum() <= max(1, n // 1000000)
    np.testing.assert_allclose(w, want_w, rtol=1e-6)


def test_mesh_sampler_is_launch_independent(cuda):
    V, F = W.torus_mesh(1.0, 0.4, 64, 32)
    a, _, _ = B.sample_points_on_mesh(5000, V, F, seed=9)
    b, _, _ = B.sample_points_on_mesh(123, V, F, seed=9)
    assert torch.equal(a[:123], b)


def test_sampled_torus_winding_number_native(cuda):
    """Config-2b style: 262,144 samples of a closed torus mesh as sources,
    2^18 queries; the native tree's winding number against the analytic
    inside/outside and the FP64 direct sum on a subset."""
    V, F = W.torus_mesh(1.0, 0.4, 128, 64)
    pts, nrm, w = B.sample_points_on_mesh(262144, V, F, seed=1)
    q = W.uniform_box_queries(1 << 18, seed=5)
    t = B.NativeTree().build(pts, w, normals=nrm, leaf_size=16, with_adjoint=False)
    wn = t.winding_number(q, beta=2.0).cpu().numpy()
    inside = W.torus_inside(q)
    d = np.abs(np.sqrt((np.sqrt(q[:, 0].astype(np.float64) ** 2 + q[:, 1] ** 2) - 1.0) ** 2 + q[:, 2] ** 2) - 0.4)
    far = d > 0.05
    assert np.abs(wn[far & inside] - 1).mean() < 0.03
    assert np.abs(wn[far & ~inside]).mean() < 0.01
    idx = np.random.default_rng(0).choice(q.shape[0], 2048, replace=False)
    want = O.direct_winding_number(pts.cpu().numpy(), nrm.cpu().numpy(), w.cpu().numpy(), q[idx])
    assert np.abs(wn[idx] - want).max() < 2e-2


def test_mesh_sampler_invalid(cuda):
    V, F = W.torus_mesh(1.0, 0.4, 8, 4)
    assert B.sample_points_on_mesh(0, V, F)[0].shape == (0, 3)
    with pytest.raises(ValueError):
        B.sample_points_on_mesh(10, V, F[:0])
    with pytest.raises(ValueError):
        B.sample_points_on_mesh(10, V[:, :2], F)
    bad = F.copy()
    bad[3, 1] = V.shape[0]  # a vertex that does not exist: the face counts as zero area
    with pytest.raises(B.SbhError):
        B.sample_points_on_mesh(10, V, bad)
    flat = np.zeros_like(V)  # no area at all
    with pytest.raises(B.SbhError):
        B.sample_points_on_mesh(10, flat, F)
    s = B.MeshSurface(V * 7.0 + 3.0, F, scale=2.0)
    p, _, _ = s.sample(4096, seed=1)
    ext = p.max(0).values - p.min(0).values
    assert float(ext.max()) <= 2.0 + 1e-5


def _perturbed_torus(seed):
    """The torus mesh with jittered vertices: a mix of acute, right-ish and
    obtuse faces."""
    V, F = W.torus_mesh(1.0, 0.4, 48, 24)
    V = V + np.random.default_rng(seed).normal(scale=0.01, size=V.shape).astype(np.float32)
    return V, F


@pytest.mark.parametrize("mesh", ["torus", "perturbed"])
def test_mesh_vertex_sources_match_oracle(cuda, mesh):
    V, F = W.torus_mesh(1.0, 0.4, 128, 64) if mesh == "torus" else _perturbed_torus(3)
    pts, nrm, m = B.mesh_vertex_sources(V, F)
    want_n, want_m = O.mesh_vertex_sources(V, F)
    assert torch.equal(pts.cpu(), torch.tensor(V))
    # FP64 sums in another order, rounded once to FP32
    np.testing.assert_allclose(m.cpu().numpy(), want_m, rtol=2e-7, atol=0)
    np.testing.assert_allclose(nrm.cpu().numpy(), want_n, rtol=0, atol=2e-7)
    area2, _ = O.mesh_face_geometry(V, F)
    assert abs(float(m.double().sum()) - 0.5 * area2.sum()) < 1e-5 * area2.sum()


def test_mesh_vertex_sources_winding_number(cuda):
    """The vertices of the closed torus mesh as winding-number sources on the
    native tree: against the FP64 direct sum of the same sources, and the
    analytic inside/outside away from the surface."""
    V, F = W.torus_mesh(1.0, 0.4, 128, 64)
    pts, nrm, m = B.MeshVertices(V, F, scale=2.8).sample()
    q = W.uniform_box_queries(1 << 16, seed=7)
    t = B.NativeTree().build(pts, m, normals=nrm, leaf_size=16, with_adjoint=False)
    wn = t.winding_number(q, beta=2.0).cpu().numpy()
    want = O.direct_winding_number(pts.cpu().numpy(), nrm.cpu().numpy(), m.cpu().numpy(), q)
    assert np.abs(wn - want).max() < 2e-2
    P = pts.cpu().numpy().astype(np.float64)
    # MeshVertices rescales the torus (extent 2.8 = 2 (R + r)) back to R 1, r 0.4
    inside = W.torus_inside(q)
    d = np.abs(np.sqrt((np.sqrt(q[:, 0].astype(np.float64) ** 2 + q[:, 1] ** 2) - 1.0) ** 2 + q[:, 2] ** 2) - 0.4)
    far = d > 0.1
    assert np.abs(P).max() <= 1.4 + 1e-6
    assert np.abs(wn[far & inside] - 1).mean() < 0.02
    assert np.abs(wn[far & ~inside]).mean() < 0.01


def test_mesh_vertex_sources_invalid(cuda):
    V, F = W.torus_mesh(1.0, 0.4, 8, 4)
    with pytest.raises(ValueError):
        B.mesh_vertex_sources(V[:, :2], F)
    bad = F.copy()
    bad[2, 0] = -1
    with pytest.raises(B.SbhError):
        B.mesh_vertex_sources(V, bad)
    # no faces: every vertex keeps mass 0 and a zero normal
    _, nrm, m = B.mesh_vertex_sources(V, F[:0])
    assert float(m.abs().max()) == 0.0 and float(nrm.abs().max()) == 0.0
