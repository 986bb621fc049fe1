"""CPU tests: the oracle (oracle/sbh_oracle.c) pinned against the reference's
own code and the known answers of the reference's tests.

* direct force / VJP vs a float64 restatement of the reference test's
  formula (python/test_jax_ffi_tree_builder.py:8-17) and torch autograd of it
  (the reference uses jax.grad, :49-86);
* the reference's CPU Tree3D + evaluateBarnesHut_stackless, compiled from its
  own headers into oracle/_ref, at beta = inf (the reference's own "exact
  direct sum via BH" idiom, python/old_interface/example.py:82-90) vs the
  oracle direct sum, and at beta = 2 vs the oracle's error expectations;
* the oracle's octree8 build invariants and its BH at large beta vs direct.
"""
import numpy as np
import pytest
import torch

import sbh_oracle as O
import sbh_workloads as W
from conftest import rel_l2


def _ref_formula(points, masses, queries, eps, cutoff):
    """Float64 restatement of _ref_softened_direct_force (test_jax_ffi_tree_builder.py:8-17)."""
    disp = queries[:, None, :] - points[None, :, :]
    r2 = (disp * disp).sum(-1)
    inv_r = 1.0 / torch.sqrt(r2 + eps * eps + 1e-12)
    inv_r3 = inv_r**3
    dist = torch.sqrt(r2 + 1e-12)
    u = dist / (2.0 * cutoff)
    att = torch.special.erfc(u) + (2.0 / np.sqrt(np.pi)) * u * torch.exp(-(u * u))
    coeff = -masses[None, :] * att * inv_r3
    return (coeff[..., None] * disp).sum(1)


def test_oracle_direct_force_matches_reference_test_formula():
    rng = np.random.default_rng(23)
    p = rng.uniform(-1, 1, (96, 3)).astype(np.float32)
    m = rng.uniform(0.1, 1.3, 96).astype(np.float32)
    q = rng.uniform(-0.7, 0.7, (31, 3)).astype(np.float32)
    got = O.direct_force_soft(p, m, q, 5e-2, 0.9)
    want = _ref_formula(torch.tensor(p, dtype=torch.float64), torch.tensor(m, dtype=torch.float64),
                        torch.tensor(q, dtype=torch.float64), 5e-2, 0.9).numpy()
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_oracle_direct_vjp_matches_autograd_of_reference_formula():
    rng = np.random.default_rng(31)
    p = rng.uniform(-1, 1, (64, 3)).astype(np.float32)
    m = rng.uniform(0.2, 1.1, 64).astype(np.float32)
    q = rng.uniform(-0.5, 0.5, (17, 3)).astype(np.float32)
    g = rng.normal(size=(17, 3)).astype(np.float32)
    got = O.direct_force_soft_vjp(p, m, q, g, 7e-2, 1.4)
    qt = torch.tensor(q, dtype=torch.float64, requires_grad=True)
    f = _ref_formula(torch.tensor(p, dtype=torch.float64), torch.tensor(m, dtype=torch.float64), qt, 7e-2, 1.4)
    (f * torch.tensor(g, dtype=torch.float64)).sum().backward()
    np.testing.assert_allclose(got, qt.grad.numpy(), rtol=1e-10, atol=1e-12)


def test_oracle_full_adjoint_matches_autograd():
    rng = np.random.default_rng(7)
    n = 48
    p = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    m = rng.uniform(0.2, 1.1, n).astype(np.float32)
    w = rng.normal(size=(n, 3)).astype(np.float32)
    eps = 0.05
    dx, dm = O.direct_full_adjoint(p, m, w, eps, 0.0)
    pt = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    mt = torch.tensor(m, dtype=torch.float64, requires_grad=True)
    disp = pt[:, None, :] - pt[None, :, :]
    r2 = (disp * disp).sum(-1)
    f = (-(mt[None, :] * (r2 + eps * eps + 1e-12) ** -1.5)[..., None] * disp).sum(1)
    (f * torch.tensor(w, dtype=torch.float64)).sum().backward()
    np.testing.assert_allclose(dx, pt.grad.numpy(), rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(dm, mt.grad.numpy(), rtol=1e-9, atol=1e-9)


def test_oracle_bruteforce_gravity_formula():
    rng = np.random.default_rng(3)
    for dim in (2, 3):
        p = rng.uniform(-1, 1, (50, dim)).astype(np.float32)
        m = rng.uniform(0.1, 1, 50).astype(np.float32)
        q = rng.uniform(-1, 1, (20, dim)).astype(np.float32)
        got = O.bruteforce_gravity(p, m, q)
        d = np.linalg.norm(p[None].astype(np.float64) - q[:, None].astype(np.float64), axis=-1)
        np.testing.assert_allclose(got, (-m[None] / (d + 0.1)).sum(1), rtol=1e-12)


@pytest.mark.skipif(not O.available("libsbh_ref_cpu.so"), reason="reference CPU build missing (make -C oracle ref)")
def test_reference_cpu_bh_at_infinite_beta_is_the_direct_sum():
    p, m = W.uniform_cube(3000, seed=4)
    for variant in (0, 2):
        for double in (False, True):
            t = O.RefTree3D(p, m, variant=variant, double=double)
            got, counts = t.eval(p[:200], 1e30, O.REF_K_SOFT_FORCE, eps=1e-3)
            want = O.direct_force_soft(p, m, p[:200], 1e-3)
            assert (counts == 3000).all()
            assert rel_l2(got, want) < (1e-12 if double else 2e-6)


@pytest.mark.skipif(not O.available("libsbh_ref_cpu.so"), reason="reference CPU build missing (make -C oracle ref)")
def test_reference_cpu_winding_number_and_vjp_at_infinite_beta():
    pts, nrm, w = W.ellipsoid_surface(2000, seed=2)
    q = W.uniform_box_queries(300, seed=3)
    t = O.RefTree3D(pts, w, normals=nrm, variant=0, double=True)
    got, _ = t.eval(q, 1e30, O.REF_K_WINDING)
    want = O.direct_winding_number(pts, nrm, w, q)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12)
    cot = np.random.default_rng(1).normal(size=(300, 3)).astype(np.float32)
    got, _ = t.eval(q, 1e30, O.REF_K_SOFT_FORCE_VJP, eps=1e-2, cot=cot)
    want = O.direct_force_soft_vjp(pts, w, q, cot, 1e-2)
    assert rel_l2(got, want) < 1e-12


def test_octree8_oracle_build_invariants_and_direct_limit():
    p, m = W.plummer(3000, seed=9)
    nrm = np.zeros_like(p)
    mn = p.min(0) - np.float32(1e-3)
    mx = p.max(0) + np.float32(1e-3)
    leaf, node, contrib, codes, perm = O.build_octree8(p, nrm, m, mn, mx, 5)
    nodes = node.view(np.uint8).reshape(-1, 104)
    start = nodes[:, 0:4].copy().view(np.uint32).ravel()
    end = nodes[:, 4:8].copy().view(np.uint32).ravel()
    mass = nodes[:, 96:100].copy().view(np.float32).ravel()
    assert start[0] == 0 and end[0] == 3000
    assert np.isclose(mass[0], m.sum(), rtol=1e-6)
    assert sorted(perm.tolist()) == list(range(3000))
    assert (np.diff(codes[perm].astype(np.int64)) >= 0).all()
    # the dense traversal at huge beta only sums leaves: the direct sum
    got, counts = O.bh_octree8(leaf, node, p[:100], 1e30, O.KERNEL_SOFT, eps=1e-3)
    want = O.direct_force_soft(p, m, p[:100], 1e-3)
    assert rel_l2(got, want) < 1e-12
