"""GPU: the native stochastic Barnes-Hut estimator (sbh_native_stochastic_force)
against the oracle's restatement (orc_native_stochastic) run on the GPU's own
exported tree: at a fixed seed both draw the same nodes, so every row agrees
within FP32 tolerance; over seeds the mean converges to the expectation, the
force walk at beta with the quadrupole everywhere (on the GPU, and the
oracle's), within its standard error; and the error against the FP64 direct
sum at 32 drawn nodes per query is bounded."""
import ctypes

import numpy as np
import pytest
import torch

import sbh_b200 as B
import sbh_oracle as O
import sbh_workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _tree(n, seed=3, leaf=16):
    p, m = W.plummer(n, seed=seed)
    t = B.NativeTree().build(p, m, leaf_size=leaf)
    _, perm, rec = t.export()
    sp = np.ascontiguousarray(np.concatenate([p[perm], m[perm, None]], axis=1), np.float32)
    return p, m, t, sp, perm, rec


@pytest.mark.parametrize("bc,K", [(1.0, 32), (1.5, 32), (1.0, 1), (0.75, 7)])
def test_fixed_seed_matches_oracle(cuda, bc, K):
    p, m, t, sp, perm, rec = _tree(20000)
    got = t.stochastic_force(beta=2.0, beta_coarse=bc, samples=K, seed=11, softening=1e-3).cpu().numpy()
    want, ex, walks = O.native_stochastic(sp, perm, rec, group_size=B.native_group_size(), beta_coarse=bc, beta=2.0,
                                          softening=1e-3, samples=K, seed=11)
    assert walks > 0
    # same draws: the rows differ by FP32 rounding of the coarse part and of
    # each drawn node's (refined - quadrupole) difference times its weight
    assert rel_l2(got, want) < 3e-5
    row = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
    assert row.max() < 2e-3, f"worst row {row.max():.2e}"
    # and the estimate is not its expectation (the draws do something)
    assert rel_l2(want, ex) > 1e-6


def test_unbiased_over_seeds(cuda):
    p, m, t, sp, perm, rec = _tree(8000, seed=4)
    S, K = 64, 4
    runs = np.stack([t.stochastic_force(beta_coarse=1.0, samples=K, seed=1000 + s).cpu().numpy().astype(np.float64)
                     for s in range(S)])
    _, ex, _ = O.native_stochastic(sp, perm, rec, group_size=B.native_group_size(), beta_coarse=1.0, samples=K,
                                   seed=0)
    # the expectation is the force walk at beta = 2 with the quadrupole everywhere
    walk = t.force(beta=2.0, softening=1e-3, quadrupole_radius=0.0, quadrupole_linear=0.0).cpu().numpy()
    assert rel_l2(walk, ex) < 1e-5
    mean, sd = runs.mean(0), runs.std(0, ddof=1)
    scale = np.linalg.norm(ex, axis=1, keepdims=True) * np.ones((1, 3))
    noisy = sd > 1e-4 * scale  # components where sampling noise dominates FP32 rounding
    assert noisy.mean() > 0.5
    # rows of one group share their draws, so z-scores of one group are
    # correlated; their mean square still has expectation 63 / 61
    z = (mean - ex)[noisy] / (sd[noisy] / np.sqrt(S))
    assert 0.7 < float(np.mean(z * z)) < 1.4, float(np.mean(z * z))
    assert float(np.mean(np.abs(z) > 5.0)) < 2e-3
    # rows without spread are deterministic and equal the expectation
    quiet = ~noisy
    assert np.all(np.abs(mean - ex)[quiet] <= 1e-4 * scale[quiet] + 1e-7)
    # the mean over 64 seeds is 8x closer to the walk than one estimate
    assert rel_l2(mean, walk) < 0.25 * rel_l2(runs[0], walk)


def test_accuracy_vs_fp64_direct(cuda):
    n = 1 << 17
    p, m = W.plummer(n, seed=5)
    t = B.NativeTree().build(p, m)
    idx = np.random.default_rng(6).choice(n, 1024, replace=False)
    ref = O.direct_force_soft(p, m, p[idx], 1e-3)
    # 32 drawn nodes per query (CPU restatement at 5e4 particles: 8.1e-4 and 1.8e-4)
    est = t.stochastic_force(samples=32, beta_coarse=1.0, seed=1).cpu().numpy()
    assert rel_l2(est[idx], ref) < 2.5e-3
    est = t.stochastic_force(samples=32, beta_coarse=1.5, seed=1).cpu().numpy()
    assert rel_l2(est[idx], ref) < 6e-4


def test_determinism_and_validation(cuda):
    p, m, t, sp, perm, rec = _tree(3000, seed=7)
    a = t.stochastic_force(seed=5)
    b = t.stochastic_force(seed=5)
    c = t.stochastic_force(seed=6)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert not torch.equal(a, c)
    # beta_coarse = beta: every weight is zero, the estimate is the force walk
    # (the same terms, summed in another order)
    d = t.stochastic_force(beta_coarse=2.0, seed=5)
    e = t.stochastic_force(beta_coarse=2.0, seed=9)
    f = t.force(beta=2.0, quadrupole_radius=0.0, quadrupole_linear=0.0)
    assert torch.equal(d, e)
    assert rel_l2(d.cpu().numpy(), f.cpu().numpy()) < 1e-6
    with pytest.raises(ValueError):
        t.stochastic_force(beta_coarse=2.5)  # coarser than beta is required
    for k in (0, 1025):
        with pytest.raises(ValueError):
            t.stochastic_force(samples=k)
    L = B.lib()
    prm = t.params(2.0, 1e-3, 0.5, False)  # an erfc cutoff: not served
    out = torch.empty((t.n, 3), device=cuda)
    s = torch.cuda.current_stream(cuda).cuda_stream
    assert L.sbh_native_stochastic_force(s, ctypes.byref(prm), 1.0, 8, ctypes.c_uint64(1), out.data_ptr(),
                                         t.ws.data_ptr(), t.ws.numel()) != 0
    assert "free-space" in B.last_error()


@pytest.mark.parametrize("bc,K", [(1.0, 8), (1.5, 32)])
def test_vjp_matches_oracle_plan_adjoint(cuda, bc, K):
    """The adjoint of the estimate with the draws held fixed: gradients with
    respect to every position and mass against the oracle's adjoint of the
    same terms (orc_native_stochastic_plan on the GPU's node records, FP64)."""
    p, m, t, sp, perm, rec = _tree(20000, seed=12)
    w = np.random.default_rng(13).normal(size=p.shape).astype(np.float32)
    f, gx, gm = t.stochastic_force_vjp(w, beta=2.0, beta_coarse=bc, samples=K, seed=5, softening=1e-3)
    est = t.stochastic_force(beta=2.0, beta_coarse=bc, samples=K, seed=5, softening=1e-3)
    torch.cuda.synchronize()
    assert torch.equal(f, est)  # the same draws
    T = O.NativeTree(p, m, leaf_size=16)
    assert T.stochastic_plan(rec, group_size=B.native_group_size(), beta_coarse=bc, beta=2.0, softening=1e-3,
                             samples=K, seed=5) > 0
    dx, dm = T.adjoint(w, 1e-3, quad=True)
    assert rel_l2(gx.cpu().numpy(), dx) < 1e-4
    assert rel_l2(gm.cpu().numpy(), dm) < 1e-4
    # the drawn terms matter: the classic walk's adjoint is farther away
    _, cx, cm = t.force_vjp(w, beta=2.0, softening=1e-3, quadrupole_radius=0.0, quadrupole_linear=0.0)
    assert rel_l2(cx.cpu().numpy(), dx) > 3 * rel_l2(gx.cpu().numpy(), dx)


def test_vjp_at_beta_coarse_equal_beta_is_the_force_walk_adjoint(cuda):
    p, m, t, sp, perm, rec = _tree(8000, seed=14)
    w = np.random.default_rng(15).normal(size=p.shape).astype(np.float32)
    _, gx, gm = t.stochastic_force_vjp(w, beta_coarse=2.0, seed=3, want_force=False)
    _, cx, cm = t.force_vjp(w, beta=2.0, softening=1e-3, quadrupole_radius=0.0, quadrupole_linear=0.0)
    assert rel_l2(gx.cpu().numpy(), cx.cpu().numpy()) < 1e-5
    assert rel_l2(gm.cpu().numpy(), cm.cpu().numpy()) < 1e-5


def test_autograd_matches_the_entry_point(cuda):
    p, m = W.plummer(6000, seed=16)
    P = torch.tensor(p, device=cuda, requires_grad=True)
    M = torch.tensor(m, device=cuda, requires_grad=True)
    f = B.native_stochastic_force(P, M, beta_coarse=1.0, samples=16, seed=9)
    w = torch.randn_like(f)
    (f * w).sum().backward()
    t = B.NativeTree().build(p, m)
    f2, gx, gm = t.stochastic_force_vjp(w, beta_coarse=1.0, samples=16, seed=9)
    torch.cuda.synchronize()
    assert torch.equal(f.detach(), f2)
    # the node-side and source-side sums are float atomics: equal up to their order
    assert rel_l2(P.grad.cpu().numpy(), gx.cpu().numpy()) < 1e-5
    assert rel_l2(M.grad.cpu().numpy(), gm.cpu().numpy()) < 1e-5


def test_forest_and_tiny_systems_match_oracle(cuda):
    """A forest of systems of 3,000, 17, 12,000 and 1 particles in one launch:
    every group walks its own system's tree, draws by its own first input
    index, and equals the oracle's restatement on the exported records; at
    beta_coarse = beta the adjoint is the force walk's."""
    systems = [W.plummer(n, seed=20 + i) for i, n in enumerate((3000, 17, 12000, 1))]
    pts = np.concatenate([s[0] + np.float32(50.0 * i) for i, s in enumerate(systems)])
    ms = np.concatenate([s[1] for s in systems])
    offs = np.cumsum([0] + [s[0].shape[0] for s in systems])
    t = B.NativeTree().build(pts, ms, system_offsets=offs, leaf_size=16)
    _, perm, rec = t.export()
    sp = np.ascontiguousarray(np.concatenate([pts[perm], ms[perm, None]], axis=1), np.float32)
    got = t.stochastic_force(beta_coarse=1.0, samples=16, seed=2).cpu().numpy()
    want, ex, walks = O.native_stochastic(sp, perm, rec, group_size=B.native_group_size(), beta_coarse=1.0,
                                          samples=16, seed=2)
    assert walks > 0 and np.isfinite(got).all()
    assert rel_l2(got, want) < 3e-5
    for i in range(len(systems)):  # per system too (the 1-particle system feels no force)
        a, b = offs[i], offs[i + 1]
        if np.abs(want[a:b]).max() > 0:
            assert rel_l2(got[a:b], want[a:b]) < 1e-4
        else:
            assert np.abs(got[a:b]).max() == 0
    w = np.random.default_rng(21).normal(size=pts.shape).astype(np.float32)
    _, gx, gm = t.stochastic_force_vjp(w, beta_coarse=2.0, want_force=False)
    _, cx, cm = t.force_vjp(w, beta=2.0, softening=1e-3, quadrupole_radius=0.0, quadrupole_linear=0.0,
                            want_force=False)
    assert rel_l2(gx.cpu().numpy(), cx.cpu().numpy()) < 1e-5
    assert rel_l2(gm.cpu().numpy(), cm.cpu().numpy()) < 1e-5


def test_empty_and_coincident_points(cuda):
    """An empty tree gives empty outputs; a cloud with 600 copies of three
    points (nodes whose particles coincide have r_g = 0 and weight 0, and
    leaves beyond the leaf size) still equals the oracle's restatement."""
    t = B.NativeTree().build(np.zeros((0, 3), np.float32), np.zeros(0, np.float32))
    assert t.stochastic_force().shape == (0, 3)
    f, gx, gm = t.stochastic_force_vjp(np.zeros((0, 3), np.float32))
    assert f.shape == (0, 3) and gx.shape == (0, 3) and gm.shape == (0,)
    p, _ = W.uniform_cube(2000, seed=31)
    p = np.concatenate([p, np.repeat(p[:3], 200, axis=0)]).astype(np.float32)
    m = np.full(p.shape[0], 1.0 / p.shape[0], np.float32)
    t = B.NativeTree().build(p, m, leaf_size=16)
    _, perm, rec = t.export()
    sp = np.ascontiguousarray(np.concatenate([p[perm], m[perm, None]], axis=1), np.float32)
    got = t.stochastic_force(beta_coarse=1.0, samples=32, seed=4).cpu().numpy()
    want, _, _ = O.native_stochastic(sp, perm, rec, group_size=B.native_group_size(), beta_coarse=1.0, samples=32,
                                     seed=4)
    assert np.isfinite(got).all()
    assert rel_l2(got, want) < 3e-5
