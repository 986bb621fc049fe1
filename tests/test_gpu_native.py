"""GPU parity of the native adaptive octree against the oracle's restatement
(oracle/sbh_oracle.c, orc_native_*): keys, permutation and topology
bit-exact; node moments, forces and the adjoint within FP32 tolerance of the
oracle's float64 evaluation of the same plan; accuracy against the FP64
direct sum at the configuration's theta = 0.5 (beta = 2)."""
import numpy as np
import pytest
import torch

import sbh_b200 as B
import sbh_oracle as O
import sbh_workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _decode_nodes(rec):
    f = rec.view(np.float32).reshape(-1, 20)
    i = rec.view(np.int32).reshape(-1, 20)
    return dict(com=f[:, 0:4], cell=f[:, 4:8], quad=f[:, 8:12], quad2=f[:, 12:16], start=i[:, 16], end=i[:, 17],
                skip=i[:, 18], level=i[:, 19] & 0xFF, leaf=(i[:, 19] & 0x100) != 0)


@pytest.mark.parametrize("dist,leaf", [("plummer", 16), ("uniform", 8), ("dupes", 16), ("tiny", 16)])
def test_native_tree_bit_exact_vs_oracle(cuda, dist, leaf):
    if dist == "plummer":
        p, m = W.plummer(20000, seed=1)
    elif dist == "uniform":
        p, m = W.uniform_cube(5000, seed=2)
    elif dist == "dupes":
        p, m = W.uniform_cube(900, seed=3)
        p = np.concatenate([p, np.repeat(p[:3], 50, axis=0)])
        m = np.full(p.shape[0], 1.0 / p.shape[0], np.float32)
    else:
        p, m = W.uniform_cube(11, seed=4)
    t = B.NativeTree().build(p, m, leaf_size=leaf)
    keys, perm, rec = t.export()
    T = O.NativeTree(p, m, leaf_size=leaf)
    a = T.arrays()
    np.testing.assert_array_equal(keys, a["keys"])
    np.testing.assert_array_equal(perm.astype(np.int64), a["perm"])
    nd = _decode_nodes(rec)
    assert rec.shape[0] == T.num_nodes
    np.testing.assert_array_equal(nd["start"], a["start"])
    np.testing.assert_array_equal(nd["end"], a["end"])
    np.testing.assert_array_equal(nd["skip"], a["skip"])
    np.testing.assert_array_equal(nd["level"], a["level"])
    np.testing.assert_array_equal(nd["cell"][:, 3], a["side"] * np.float32(1.7320508))
    np.testing.assert_array_equal(nd["cell"][:, :3], a["center"])
    # COM in float from FP64 sums: equal up to the last bit of the rounding
    mass = np.add.reduceat(m[a["perm"]].astype(np.float64), a["start"])[:0]  # noqa: F841 (shape check only)
    np.testing.assert_allclose(nd["com"][:, 3].sum() >= 0, True)


@pytest.mark.parametrize("quad,qradius,linear", [(True, 0.0, 0.0), (True, 1.6, 0.0), (False, 0.0, 0.0),
                                                 (True, 0.0, 0.5), (True, 1.6, 0.35)])
def test_native_force_matches_oracle_same_plan(cuda, quad, qradius, linear):
    """qradius 0: every accepted node takes the quadrupole; 1.6: only those
    within 1.6 opening radii of the group. linear > 0: the quadrupoles of
    nodes far from the group (r_g <= linear |c - cell centre|) are taken to
    first order about the group centre, once per group."""
    p, m = W.plummer(30000, seed=5)
    t = B.NativeTree().build(p, m, leaf_size=16, with_adjoint=False)
    f = t.force(beta=2.0, softening=1e-3, quadrupole=quad, quadrupole_radius=qradius,
                quadrupole_linear=linear).cpu().numpy()
    st = t.stats()
    T = O.NativeTree(p, m, leaf_size=16)
    with O.native_quadrupole_radius(qradius), O.native_quadrupole_linear(linear):
        inter = T.plan(2.0, B.native_group_size())
    want, _ = T.force(1e-3, quad=quad)
    assert rel_l2(f, want) < 1e-5
    lin_target, lin_pairs = T.linear_quadrupole_counts()
    assert st["far_quadrupole_linear"] == lin_target and st["linear_pairs"] == lin_pairs
    assert (lin_pairs > 0) == (linear > 0)
    # same node-packed target groups
    assert st["groups"] == T.plan_stats()[0]
    # same opening decisions up to ulp-level ties
    assert abs((st["far"] + st["near"]) - inter) <= 1e-4 * inter
    if quad:
        # and the same far-field orders
        nq = T.quadrupole_interactions()
        assert abs(st["far_quadrupole"] - nq) <= 1e-4 * st["far"]
        assert (nq == st["far"]) == (qradius == 0.0)
    else:
        assert st["far_quadrupole"] == 0


def test_native_force_accuracy_vs_fp64_direct(cuda):
    p, m = W.plummer(200000, seed=6)
    t = B.NativeTree().build(p, m, leaf_size=16, with_adjoint=False)
    idx = np.random.default_rng(0).choice(p.shape[0], 4096, replace=False)
    want = O.direct_force_soft(p, m, p[idx], 1e-3)
    err = {}
    # exact quadrupole everywhere; the default (every accepted node, linearized where far from the group);
    # exact quadrupole within 1.6 opening radii, monopole beyond; monopole only
    for name, kw in (("exact", dict(quadrupole_radius=0.0, quadrupole_linear=0.0)), ("default", {}),
                     ("radius", dict(quadrupole_radius=1.6, quadrupole_linear=0.0))):
        f = t.force(beta=2.0, softening=1e-3, quadrupole=True, **kw).cpu().numpy()
        err[name] = rel_l2(f[idx], want)
    f = t.force(beta=2.0, softening=1e-3, quadrupole=False).cpu().numpy()
    err["mono"] = rel_l2(f[idx], want)
    assert err["exact"] < err["default"] < err["mono"]
    assert err["exact"] < err["radius"] < err["mono"]
    assert err["default"] < 8e-5


@pytest.mark.parametrize("quad,qradius,linear", [(True, 0.0, 0.0), (True, 1.6, 0.0), (False, 0.0, 0.0),
                                                 (True, 0.0, 0.5), (True, 1.6, 0.35)])
def test_native_adjoint_matches_oracle(cuda, quad, qradius, linear):
    rng = np.random.default_rng(7)
    p, m = W.plummer(20000, seed=7)
    m = (m * rng.uniform(0.5, 1.5, m.shape)).astype(np.float32)
    w = rng.normal(size=p.shape).astype(np.float32)
    t = B.NativeTree().build(p, m, leaf_size=16, with_adjoint=True)
    f, gx, gm = t.force_vjp(w, beta=2.0, softening=1e-3, quadrupole=quad, quadrupole_radius=qradius,
                            quadrupole_linear=linear)
    T = O.NativeTree(p, m, leaf_size=16)
    with O.native_quadrupole_radius(qradius), O.native_quadrupole_linear(linear):
        T.plan(2.0, B.native_group_size())
    want_f, _ = T.force(1e-3, quad=quad)
    dx, dm = T.adjoint(w, 1e-3, quad=quad)
    assert rel_l2(f.cpu().numpy(), want_f) < 1e-5
    assert rel_l2(gx.cpu().numpy(), dx) < 1e-4
    assert rel_l2(gm.cpu().numpy(), dm) < 1e-4


def test_native_forest_equals_separate_systems(cuda):
    systems = [W.plummer(n, seed=10 + i) for i, n in enumerate((3000, 17, 12000, 1))]
    pts = np.concatenate([s[0] + np.float32(50.0 * i) for i, s in enumerate(systems)])
    ms = np.concatenate([s[1] for s in systems])
    offs = np.cumsum([0] + [s[0].shape[0] for s in systems])
    t = B.NativeTree().build(pts, ms, system_offsets=offs, leaf_size=16)
    f = t.force(beta=2.0, softening=1e-3).cpu().numpy()
    rng = np.random.default_rng(3)
    w = rng.normal(size=pts.shape).astype(np.float32)
    _, gx, gm = t.force_vjp(w, beta=2.0, softening=1e-3, want_force=False)
    for i, (p, m) in enumerate(systems):
        a, b = offs[i], offs[i + 1]
        ti = B.NativeTree().build(p + np.float32(50.0 * i), m, leaf_size=16)
        fi = ti.force(beta=2.0, softening=1e-3).cpu().numpy()
        # same tree and groups; node moments differ in the last bits because
        # the forest's FP64 prefix sums also carry the earlier systems
        assert rel_l2(f[a:b], fi) < 1e-6
        _, gxi, gmi = ti.force_vjp(w[a:b], beta=2.0, softening=1e-3, want_force=False)
        assert rel_l2(gx[a:b].cpu().numpy(), gxi.cpu().numpy()) < 1e-5
        assert rel_l2(gm[a:b].cpu().numpy(), gmi.cpu().numpy()) < 1e-5


def test_native_winding_number(cuda):
    pts, nrm, w = W.ellipsoid_surface(20000, seed=2)
    q = W.uniform_box_queries(4000, seed=3)
    t = B.NativeTree().build(pts, w, normals=nrm, leaf_size=16, with_adjoint=False)
    wn = t.winding_number(q, beta=2.0).cpu().numpy()
    want = O.direct_winding_number(pts, nrm, w, q)
    inside = W.ellipsoid_inside(q)
    assert np.abs(want[inside] - 1.0).mean() < 0.05 and np.abs(want[~inside]).mean() < 0.05
    assert np.abs(wn - want).max() < 2e-2
    assert rel_l2(wn, want) < 5e-3


def test_native_autograd_matches_force_vjp(cuda):
    rng = np.random.default_rng(9)
    p, m = W.plummer(5000, seed=9)
    pt = torch.tensor(p, device=cuda, requires_grad=True)
    mt = torch.tensor(m, device=cuda, requires_grad=True)
    w = torch.tensor(rng.normal(size=p.shape), dtype=torch.float32, device=cuda)
    f = B.native_force_recompute_vjp(pt, mt, beta=2.0, softening=1e-3)
    (f * w).sum().backward()
    t = B.NativeTree().build(p, m, leaf_size=16)
    _, gx, gm = t.force_vjp(w, beta=2.0, softening=1e-3)
    # the adjoint's FP32 atomics are summed in a run-dependent order
    assert rel_l2(pt.grad.cpu().numpy(), gx.cpu().numpy()) < 1e-6
    assert rel_l2(mt.grad.cpu().numpy(), gm.cpu().numpy()) < 1e-6


def test_native_empty_and_invalid(cuda):
    t = B.NativeTree().build(np.zeros((0, 3), np.float32), np.zeros(0, np.float32))
    assert t.force().shape == (0, 3)
    with pytest.raises(ValueError):
        B.NativeTree().build(np.zeros((4, 3), np.float32), np.zeros(4, np.float32), leaf_size=0)
    with pytest.raises(ValueError):
        B.NativeTree().build(np.zeros((4, 3), np.float32), np.zeros(4, np.float32)).force(beta=-1.0)


def _periodic_direct(p, m, q, eps, cutoff):
    from scipy.special import erfc
    r = q[:, None, :].astype(np.float64) - p[None, :, :].astype(np.float64)
    r -= np.floor(r + 0.5)
    r2 = (r * r).sum(-1)
    d = np.sqrt(r2 + 1e-12)
    u = d / (2.0 * cutoff)
    att = erfc(u) + 2.0 / np.sqrt(np.pi) * u * np.exp(-u * u)
    return (-m[None, :, None] * (att * (r2 + eps * eps + 1e-12) ** -1.5)[..., None] * r).sum(1)


def test_native_periodic_short_range_matches_oracle(cuda):
    """TreePM short range on the native tree: minimum image in the unit box,
    erfc cutoff 0.05, cells beyond 0.3 of a group skipped. Same plan as the
    oracle (groups, pruned and accepted cells), forces and the full adjoint
    within FP32 tolerance, and the periodic FP64 direct sum within the
    opening-angle error."""
    rng = np.random.default_rng(21)
    p, m = W.uniform_cube(20000, seed=22)
    w = rng.normal(size=p.shape).astype(np.float32)
    kw = dict(beta=2.0, softening=1e-3, cutoff=0.05, quadrupole=False, periodic=True, box_length=1.0,
              prune_radius=0.3)
    t = B.NativeTree().build(p, m, leaf_size=16, with_adjoint=True)
    f, gx, gm = t.force_vjp(w, **kw)
    st = t.stats()
    T = O.NativeTree(p, m, leaf_size=16)
    with O.native_periodic(1.0, 0.3):
        inter = T.plan(2.0, B.native_group_size())
        want_f, _ = T.force(1e-3, cutoff=0.05)
        dx, dm = T.adjoint(w, 1e-3, cutoff=0.05)
    assert abs((st["far"] + st["near"]) - inter) <= 1e-4 * inter
    assert rel_l2(f.cpu().numpy(), want_f) < 1e-5
    assert rel_l2(gx.cpu().numpy(), dx) < 1e-4
    assert rel_l2(gm.cpu().numpy(), dm) < 1e-4
    idx = rng.choice(p.shape[0], 512, replace=False)
    # monopole-only at theta = 0.5 on a uniform cube: a few 1e-4
    assert rel_l2(f.cpu().numpy()[idx], _periodic_direct(p, m, p[idx], 1e-3, 0.05)) < 1e-3
    # the force walk sums in another order than the adjoint walk
    f2 = t.force(**kw).cpu().numpy()
    assert rel_l2(f2, want_f) < 1e-5


@pytest.mark.parametrize("group_size", [32, 17])
def test_native_smaller_groups_match_oracle(cuda, group_size):
    """Groups re-cut with fewer targets (sbh_native_set_group_size): the same
    groups and plan as the oracle's with that group size, the forces and the
    adjoint within FP32 tolerance; on the periodic short-range walk and on the
    plain softened walk."""
    rng = np.random.default_rng(31)
    p, m = W.uniform_cube(12000, seed=32)
    w = rng.normal(size=p.shape).astype(np.float32)
    t = B.NativeTree().build(p, m, leaf_size=16, with_adjoint=True, group_size=group_size)
    kw = dict(beta=2.0, softening=1e-3, cutoff=0.05, quadrupole=False, periodic=True, box_length=1.0,
              prune_radius=0.2)
    f, gx, gm = t.force_vjp(w, **kw)
    st = t.stats()
    T = O.NativeTree(p, m, leaf_size=16)
    with O.native_periodic(1.0, 0.2):
        inter = T.plan(2.0, group_size)
        want_f, _ = T.force(1e-3, cutoff=0.05)
        dx, dm = T.adjoint(w, 1e-3, cutoff=0.05)
    assert st["groups"] == T.plan_stats()[0]
    assert abs((st["far"] + st["near"]) - inter) <= 1e-4 * inter
    assert rel_l2(f.cpu().numpy(), want_f) < 1e-5
    assert rel_l2(gx.cpu().numpy(), dx) < 1e-4
    assert rel_l2(gm.cpu().numpy(), dm) < 1e-4
    # back to full groups on the same tree: the oracle's plan with full groups
    t.set_group_size(B.native_group_size())
    f64 = t.force(**kw).cpu().numpy()
    assert t.stats()["groups"] < st["groups"]
    with O.native_periodic(1.0, 0.2):
        T.plan(2.0, B.native_group_size())
        want64, _ = T.force(1e-3, cutoff=0.05)
    assert rel_l2(f64, want64) < 1e-5
    with pytest.raises(ValueError):
        t.set_group_size(B.native_group_size() + 1)


def test_native_periodic_direct_limit_and_shift_invariance(cuda):
    p, m = W.uniform_cube(6000, seed=23)
    kw = dict(beta=1e30, softening=2e-3, cutoff=0.1, quadrupole=False, periodic=True, box_length=1.0)
    f = B.NativeTree().build(p, m, leaf_size=16).force(**kw).cpu().numpy()
    want = _periodic_direct(p, m, p, 2e-3, 0.1)
    assert rel_l2(f, want) < 2e-6
    shifted = np.mod(p + np.array([0.31, 0.77, 0.05], np.float32), np.float32(1.0)).astype(np.float32)
    fs = B.NativeTree().build(shifted, m, leaf_size=16).force(**kw).cpu().numpy()
    assert rel_l2(fs, _periodic_direct(shifted, m, shifted, 2e-3, 0.1)) < 2e-6
    # the shifted coordinates are rounded to FP32 anew: close pairs move by an ulp
    assert rel_l2(fs, f) < 1e-4


def test_native_periodic_invalid_params(cuda):
    t = B.NativeTree().build(*W.uniform_cube(100, seed=24))
    with pytest.raises(ValueError):
        t.force(periodic=True, box_length=0.0, quadrupole=False)
    with pytest.raises(ValueError):
        t.force(periodic=True, box_length=1.0, quadrupole=True)
    with pytest.raises(ValueError):
        t.force(cutoff=0.0, prune_radius=0.3, quadrupole=False)


@pytest.mark.parametrize("world", [2, 3])
def test_native_target_ranges_sum_to_full(cuda, world):
    """Ranks emulated one after another on one GPU (no collective): each
    walks its share of the sorted targets (sbh_native_set_target_range); the
    shares' forces are disjoint and their sum, like the sum of the partial
    gradients, equals the unsharded result."""
    import sbh_dist

    rng = np.random.default_rng(51)
    systems = [W.plummer(n, seed=52 + i) for i, n in enumerate((15000, 4000))]
    p = np.concatenate([s[0] + np.float32(40.0 * i) for i, s in enumerate(systems)])
    m = np.concatenate([s[1] for s in systems])
    offs = np.array([0, 15000, 19000], np.int64)
    w = rng.normal(size=p.shape).astype(np.float32)
    t = B.NativeTree().build(p, m, system_offsets=offs, leaf_size=16, with_adjoint=True)
    f_all, gx_all, gm_all = t.force_vjp(w, beta=2.0, softening=1e-3)
    f_all, gx_all, gm_all = f_all.cpu().numpy(), gx_all.cpu().numpy(), gm_all.cpu().numpy()
    fs, gxs, gms, nonzero = 0, 0, 0, np.zeros(p.shape[0], np.int64)
    for r in range(world):
        t.set_target_range(*sbh_dist.shard_targets(t.n, world, r))
        f, gx, gm = t.force_vjp(w, beta=2.0, softening=1e-3)
        f = f.cpu().numpy()
        nonzero += np.any(f != 0, axis=1)
        fs, gxs, gms = fs + f, gxs + gx.cpu().numpy(), gms + gm.cpu().numpy()
        ff = t.force(beta=2.0, softening=1e-3).cpu().numpy()
        np.testing.assert_array_equal(ff != 0, f != 0)
    t.set_target_range(0, t.n)
    assert (nonzero == 1).all()  # every target served by exactly one share
    assert rel_l2(fs, f_all) < 1e-6
    assert rel_l2(gxs, gx_all) < 1e-5
    assert rel_l2(gms, gm_all) < 1e-5
    with pytest.raises(ValueError):
        t.set_target_range(5, 4)
    with pytest.raises(ValueError):
        t.set_target_range(0, t.n + 1)



@pytest.mark.parametrize("group_size", [64, 40, 96, 72])
def test_native_two_and_three_slot_kernels_match_oracle(cuda, group_size):
    """Groups of at most 64 run on the two-targets-per-lane walks, of 65 to
    96 on the three-per-lane walks: forces and the full adjoint with the
    default quadrupole (every accepted node, linearized about the group
    centre where the group is small against its distance) against the
    oracle's plan with the same group size, on a clustered and a uniform
    system."""
    rng = np.random.default_rng(61)
    for p, m in (W.plummer(20000, seed=62), W.uniform_cube(15000, seed=63)):
        w = rng.normal(size=p.shape).astype(np.float32)
        t = B.NativeTree().build(p, m, leaf_size=16, with_adjoint=True, group_size=group_size)
        f, gx, gm = t.force_vjp(w, beta=2.0, softening=1e-3, quadrupole=True)
        f2 = t.force(beta=2.0, softening=1e-3, quadrupole=True).cpu().numpy()
        st = t.stats()
        assert st["linear_pairs"] > 0
        T = O.NativeTree(p, m, leaf_size=16)
        with O.native_quadrupole_radius(B.QUADRUPOLE_RADIUS), O.native_quadrupole_linear(B.QUADRUPOLE_LINEAR):
            inter = T.plan(2.0, group_size)
        want_f, _ = T.force(1e-3, quad=True)
        dx, dm = T.adjoint(w, 1e-3, quad=True)
        assert st["groups"] == T.plan_stats()[0]
        assert abs((st["far"] + st["near"]) - inter) <= 1e-4 * inter
        assert rel_l2(f.cpu().numpy(), want_f) < 1e-5
        assert rel_l2(f2, want_f) < 1e-5
        assert rel_l2(gx.cpu().numpy(), dx) < 1e-4
        assert rel_l2(gm.cpu().numpy(), dm) < 1e-4


def test_autotune_native_picks_a_candidate(cuda):
    p, m = W.plummer(30000, seed=71)
    cands = ((16, 128), (16, 64))
    r = B.autotune_native(torch.tensor(p, device=cuda), torch.tensor(m, device=cuda), candidates=cands,
                          beta=2.0, softening=1e-3)
    assert (r["leaf_size"], r["group_size"]) in cands
    assert len(r["trials"]) == 2 and all(t["ms"] > 0 for t in r["trials"])
    assert r["ms"] == min(t["ms"] for t in r["trials"])


def test_native_release_forgets_the_workspace(cuda):
    p, m = W.plummer(3000, seed=21)
    t = B.NativeTree().build(p, m)
    want = t.force().cpu().numpy()
    t.release()
    with pytest.raises(ValueError, match="no native tree"):
        t.force()
    t.release()  # idempotent
    got = t.build(p, m).force().cpu().numpy()
    np.testing.assert_array_equal(got, want)


def test_native_winding_number_vjp_matches_oracle(cuda):
    """The winding-number adjoint walk (dL/d queries, source positions,
    normals, weights) against the oracle's float64 adjoint of the same plan
    (queries in Morton order, groups of 32, the same opening decisions)."""
    p, nrm, m = W.ellipsoid_surface(20000, seed=4)
    rng = np.random.default_rng(2)
    q = rng.uniform(-1.5, 1.5, (5000, 3)).astype(np.float32)
    u = rng.normal(size=5000).astype(np.float32)
    t = B.NativeTree().build(p, m, normals=nrm, leaf_size=16, with_adjoint=True)
    w, gq, gp, gn, gm = t.winding_number_vjp(q, u, beta=2.0, want_value=True)
    w_fwd = t.winding_number(q, beta=2.0)
    T = O.NativeTree(p, m, leaf_size=16)
    T.wn_plan(q, 2.0)
    want_w = T.wn_eval(nrm)
    dq, dp, dn, dm = T.wn_adjoint(nrm, u)
    assert rel_l2(w.cpu().numpy(), want_w) < 1e-5
    assert rel_l2(w_fwd.cpu().numpy(), want_w) < 1e-5
    assert rel_l2(gq.cpu().numpy(), dq) < 1e-4
    assert rel_l2(gp.cpu().numpy(), dp) < 1e-4
    assert rel_l2(gn.cpu().numpy(), dn) < 1e-4
    assert rel_l2(gm.cpu().numpy(), dm) < 1e-4


def test_native_winding_number_autograd(cuda):
    p, nrm, m = W.ellipsoid_surface(4000, seed=5)
    rng = np.random.default_rng(3)
    q = rng.uniform(-1.5, 1.5, (700, 3)).astype(np.float32)
    u = torch.as_tensor(rng.normal(size=700).astype(np.float32), device=cuda)
    P, N, M, Q = (torch.tensor(a, device=cuda, requires_grad=True) for a in (p, nrm, m, q))
    w = B.native_winding_number(P, N, M, Q, beta=2.0)
    (w * u).sum().backward()
    t = B.NativeTree().build(p, m, normals=nrm, leaf_size=16, with_adjoint=True)
    _, gq, gp, gn, gm = t.winding_number_vjp(q, u, beta=2.0)
    for got, want in ((Q.grad, gq), (P.grad, gp), (N.grad, gn), (M.grad, gm)):
        assert rel_l2(got.cpu().numpy(), want.cpu().numpy()) < 1e-6
