"""Query-side VJPs of the tree and octree8 targets, and the statistics of the
stochastic (MLPCV) estimators.

* The analytic VJPs that replace the reference's finite-difference wrappers
  (python/jax_sbh_ffi.py:1037-1395) equal the float64 direct-sum VJP in the
  direct limit (beta -> infinity opens every internal node), and the
  monopole VJP of the root cell when the root is accepted.
* The stochastic estimators (src/sbh_ffi.cu:2146-2442,
  include/tree_sampler_gpu.h:25-140) and their VJPs are unbiased: the mean
  over many independent draws (seeds for octree8; copies of the queries in
  different blocks for the tree sampler) agrees with the exact sum within
  its standard error.
* For a fixed seed, the stochastic VJP is the derivative of the fixed-seed
  forward wherever a small step does not flip a sampled decision.
* The stochastic recompute wrappers give the explicit fixed-seed VJP."""
from math import pi, sqrt

import numpy as np
import pytest
import torch
from scipy.special import erfc

import sbh_b200 as B
import sbh_oracle as O
import sbh_workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


# --- float64 direct sums of the reference's pair kernels -------------------
def _diff(p, q):
    return q[:, None, :].astype(np.float64) - p[None, :, :].astype(np.float64)


def _grav_grad(p, m, q):
    r = _diff(p, q)
    d = np.sqrt((r * r).sum(-1))
    return (-m[None, :, None] * r / (d[..., None] + 0.1) ** 3).sum(1)


def _grav_grad_vjp(p, m, q, g):
    r = _diff(p, q)
    d = np.sqrt((r * r).sum(-1) + 1e-12)
    den = d + 0.1
    rg = (r * g[:, None, :]).sum(-1)
    t = g[:, None, :] / den[..., None] ** 3 - (3.0 * rg / (d * den ** 4))[..., None] * r
    return (-m[None, :, None] * t).sum(1)


def _attenuation(r2, cutoff):
    dist = np.sqrt(r2 + 1e-12)
    u = dist / (2.0 * cutoff)
    e = np.exp(-u * u)
    return dist, e, erfc(u) + 2.0 / sqrt(pi) * u * e


def _soft_force(p, m, q, eps, cutoff):
    r = _diff(p, q)
    r2 = (r * r).sum(-1)
    ir = (r2 + eps * eps + 1e-12) ** -0.5
    _, _, att = _attenuation(r2, cutoff)
    return (-m[None, :, None] * (att * ir ** 3)[..., None] * r).sum(1)


def _soft_vjp(p, m, q, g, eps, cutoff):
    r = _diff(p, q)
    r2 = (r * r).sum(-1)
    ir = (r2 + eps * eps + 1e-12) ** -0.5
    dist, e, att = _attenuation(r2, cutoff)
    cc = ir ** 3 * dist * e / (2.0 * sqrt(pi) * cutoff ** 3)
    rg = (r * g[:, None, :]).sum(-1)
    t = (att * ir ** 3)[..., None] * g[:, None, :] - (rg * (3.0 * att * ir ** 5 + cc))[..., None] * r
    return (-m[None, :, None] * t).sum(1)


def _u8(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), device=dev, dtype=torch.uint8)


def _ref_tree(dim, p, m):
    if dim == 3:
        return O.RefTree3D(p, m, variant=2)
    return O.RefTree2D(p, m)


def _zcheck(samples, exact):
    """|mean - exact| of the samples in units of the mean's standard error
    (with a small floor for entries the estimator computes exactly)."""
    mean = samples.mean(0)
    se = samples.std(0, ddof=1) / np.sqrt(samples.shape[0])
    floor = 1e-5 * np.abs(exact).max()
    return np.abs(mean - exact) / (se + floor)


def _fd_rows(fwd, q, g, h=1e-3):
    """Central differences of sum(g . fwd(q)) per query row."""
    out = np.zeros(q.shape, np.float64)
    for a in range(q.shape[1]):
        e = np.zeros(q.shape[1], np.float32)
        e[a] = h
        fp = fwd(q + e).cpu().numpy().astype(np.float64)
        fm = fwd(q - e).cpu().numpy().astype(np.float64)
        out[:, a] = ((fp - fm) * g).sum(1) / (2 * h)
    return out


# --- deterministic VJPs ------------------------------------------------------
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("softened", [False, True])
def test_tree_vjp_direct_limit(cuda, dim, softened):
    p, m = W.uniform_cube(1500, seed=31)
    p = p[:, :dim].copy()
    t = _ref_tree(dim, p, m)
    leaf, node = _u8(t.leaf_bytes(), cuda), _u8(t.node_bytes(), cuda)
    rng = np.random.default_rng(4)
    q = rng.uniform(-0.2, 1.2, (300, dim)).astype(np.float32)
    g = rng.normal(size=q.shape).astype(np.float32)
    if softened:
        got = B.softened_barnes_hut_force_vjp(leaf, node, q, g, beta=1e30, softening_scale=5e-2, cutoff_scale=1.5,
                                              threads=64).cpu().numpy()
        want = _soft_vjp(p, m, q, g, 5e-2, 1.5)
    else:
        got = B.barnes_hut_force_vjp(leaf, node, q, g, beta=1e30, threads=64).cpu().numpy()
        want = _grav_grad_vjp(p, m, q, g)
    assert rel_l2(got, want) < 2e-5


def test_tree_vjp_far_root_is_the_root_monopole(cuda):
    p, m = W.plummer(4000, seed=12)
    leaf, node, contrib = B.build_octree_buffers_with_contrib(p, np.zeros_like(p), m)
    c = contrib.cpu().numpy().reshape(-1, 32)[:1].copy().view(np.float32)  # root: pos, normal, mass, alpha
    rng = np.random.default_rng(5)
    d = rng.normal(size=(200, 3))
    q = (400.0 * d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    g = rng.normal(size=q.shape).astype(np.float32)
    got = B.softened_barnes_hut_force_vjp(leaf, node, q, g, beta=2.0, softening_scale=1e-2, cutoff_scale=1e6,
                                          threads=64).cpu().numpy()
    assert rel_l2(got, _soft_vjp(c[:, :3], c[:, 6], q, g, 1e-2, 1e6)) < 1e-5
    got = B.barnes_hut_force_vjp(leaf, node, q, g, beta=2.0, threads=64).cpu().numpy()
    assert rel_l2(got, _grav_grad_vjp(c[:, :3], c[:, 6], q, g)) < 1e-5


def test_octree8_vjp_direct_limit_and_fd(cuda):
    p, m = W.uniform_cube(2000, seed=33)
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, max_depth=4)
    rng = np.random.default_rng(6)
    q = rng.uniform(-0.2, 1.2, (256, 3)).astype(np.float32)
    g = rng.normal(size=q.shape).astype(np.float32)
    got = B.barnes_hut_force_octree8_vjp(leaf, node, q, g, beta=1e30).cpu().numpy()
    assert rel_l2(got, _grav_grad_vjp(p, m, q, g)) < 2e-5
    # at beta = 2 the VJP is the derivative of the forward for fixed decisions
    got = B.barnes_hut_force_octree8_vjp(leaf, node, q, g, beta=2.0).cpu().numpy()
    fd = _fd_rows(lambda x: B.barnes_hut_force_octree8(leaf, node, x, beta=2.0), q, g)
    row = np.linalg.norm(fd - got, axis=1) / np.maximum(np.linalg.norm(got, axis=1), 1e-30)
    assert np.median(row) < 1e-2 and (row < 5e-2).mean() > 0.9


# --- stochastic estimators: unbiased over seeds -----------------------------
@pytest.mark.parametrize("softened", [False, True])
@pytest.mark.parametrize("vjp", [False, True])
def test_octree8_stochastic_unbiased_over_seeds(cuda, softened, vjp):
    # depth 6: the depth-3 subdomains have subtrees for the sampled walks to
    # descend (at depth 4 every walk reaches the leaves with probability 1
    # and the estimate is exact for every seed)
    p, m = W.uniform_cube(3000, seed=41)
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, max_depth=6)
    rng = np.random.default_rng(7)
    q = rng.uniform(0.0, 1.0, (96, 3)).astype(np.float32)
    g = rng.normal(size=q.shape).astype(np.float32)
    kw = dict(beta=1.0, samples_per_subdomain=4)
    if softened:
        kw.update(softening_scale=2e-2, cutoff_scale=1e6, prune_enabled=False)
        fn = B.softened_stochastic_barnes_hut_force_octree8_vjp if vjp else B.softened_stochastic_barnes_hut_force_octree8
        exact = _soft_vjp(p, m, q, g, 2e-2, 1e6) if vjp else _soft_force(p, m, q, 2e-2, 1e6)
    else:
        fn = B.stochastic_barnes_hut_force_octree8_vjp if vjp else B.stochastic_barnes_hut_force_octree8
        exact = _grav_grad_vjp(p, m, q, g) if vjp else _grav_grad(p, m, q)
    args = (leaf, node, q, g) if vjp else (leaf, node, q)
    samples = torch.stack([fn(*args, seed=seed, **kw) for seed in range(256)]).cpu().numpy().astype(np.float64)
    z = _zcheck(samples, exact)
    assert z.mean() < 1.5 and (z > 5).mean() < 0.01
    assert samples.std(0).max() > 0  # the estimator does sample


@pytest.mark.parametrize("dim", [2, 3])
def test_tree_mlpcv_and_its_vjp_unbiased(cuda, dim):
    """The tree sampler draws its particles from a stream seeded by the block
    index (include/tree_sampler_gpu.h:40-42, shared by the block's queries),
    so the seed alone redraws only the descent decisions. 256 copies of each
    query sit in 256 different blocks, which averages over both streams."""
    p, m = W.uniform_cube(1500, seed=43)
    p = p[:, :dim].copy()
    t = _ref_tree(dim, p, m)
    leaf, node, contrib = _u8(t.leaf_bytes(), cuda), _u8(t.node_bytes(), cuda), _u8(t.contrib_bytes(), cuda)
    rng = np.random.default_rng(8)
    q = rng.uniform(0.0, 1.0, (96, dim)).astype(np.float32)
    g = rng.normal(size=q.shape).astype(np.float32)
    copies = 256
    qq, gg = np.tile(q, (copies, 1)), np.tile(g, (copies, 1))
    kw = dict(samples_per_subdomain=2, seed=11, threads=64)
    fs = B.stochastic_barnes_hut_force(leaf, node, contrib, qq, **kw).cpu().numpy().astype(np.float64)
    vs = B.stochastic_barnes_hut_force_vjp(leaf, node, contrib, qq, gg, **kw).cpu().numpy().astype(np.float64)
    for samples, exact in ((fs, _grav_grad(p, m, q)), (vs, _grav_grad_vjp(p, m, q, g))):
        z = _zcheck(samples.reshape(copies, 96, dim), exact)
        assert z.mean() < 1.5 and (z > 5).mean() < 0.01


def test_tree_mlpcv_vjp_is_the_fixed_seed_derivative(cuda):
    p, m = W.uniform_cube(1500, seed=45)
    t = _ref_tree(3, p, m)
    leaf, node, contrib = _u8(t.leaf_bytes(), cuda), _u8(t.node_bytes(), cuda), _u8(t.contrib_bytes(), cuda)
    rng = np.random.default_rng(9)
    q = rng.uniform(0.0, 1.0, (128, 3)).astype(np.float32)
    g = rng.normal(size=q.shape).astype(np.float32)
    kw = dict(samples_per_subdomain=2, seed=3, softening_scale=2e-2, cutoff_scale=1e6, threads=64)
    got = B.softened_stochastic_barnes_hut_force_vjp(leaf, node, contrib, q, g, **kw).cpu().numpy()
    fd = _fd_rows(lambda x: B.softened_stochastic_barnes_hut_force(leaf, node, contrib, x, **kw), q, g)
    row = np.linalg.norm(fd - got, axis=1) / np.maximum(np.linalg.norm(got, axis=1), 1e-30)
    assert np.median(row) < 1e-2 and (row < 5e-2).mean() > 0.8


@pytest.mark.parametrize("softened", [False, True])
def test_stochastic_octree8_recompute_vjp_matches_explicit(cuda, softened):
    p, m = W.plummer(2000, seed=47)
    rng = np.random.default_rng(10)
    w = torch.tensor(rng.normal(size=p.shape), dtype=torch.float32, device=cuda)
    pt = torch.tensor(p, device=cuda, requires_grad=True)
    mt = torch.tensor(m, device=cuda, requires_grad=True)
    kw = dict(beta=1.0, samples_per_subdomain=2, seed=5)
    if softened:
        kw.update(softening_scale=1e-2, cutoff_scale=1.0)
        f = B.softened_stochastic_barnes_hut_force_octree8_recompute_vjp(pt, mt, max_depth=5, **kw)
    else:
        f = B.stochastic_barnes_hut_force_octree8_recompute_vjp(pt, mt, max_depth=5, **kw)
    (f * w).sum().backward()
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, max_depth=5)
    if softened:
        fwd = B.softened_stochastic_barnes_hut_force_octree8(leaf, node, p, **kw)
        want = B.softened_stochastic_barnes_hut_force_octree8_vjp(leaf, node, p, w, **kw)
    else:
        fwd = B.stochastic_barnes_hut_force_octree8(leaf, node, p, **kw)
        want = B.stochastic_barnes_hut_force_octree8_vjp(leaf, node, p, w, **kw)
    np.testing.assert_array_equal(f.detach().cpu().numpy(), fwd.cpu().numpy())
    np.testing.assert_array_equal(pt.grad.cpu().numpy(), want.cpu().numpy())
    assert float(mt.grad.abs().max()) == 0.0
