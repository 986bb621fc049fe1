"""CPU tests of the native-tree restatement in the oracle: topology
invariants, the infinite-beta direct limit, and the adjoint (query side,
direct sources, and the chain rule through node mass, centroid and second
moment) against central finite differences of the same frozen-plan forward
in float64."""
import numpy as np
import pytest

import sbh_oracle as O
import sbh_workloads as W
from conftest import rel_l2


def _topology_invariants(T):
    a = T.arrays()
    start, end, skip, level = a["start"], a["end"], a["skip"], a["level"]
    nn = T.num_nodes
    n = T.points.shape[0]
    assert start[0] == 0 and end[0] == n and skip[0] == nn
    leaf = (np.arange(nn) + 1 >= nn) | (skip == np.arange(nn) + 1)
    # pre-order: a child starts where its parent starts or later, inside it
    for k in range(1, nn):
        assert skip[k] > k
    assert ((end - start)[leaf & (level < 21)] <= T.leaf_size).all()
    assert ((end - start)[~leaf] > T.leaf_size).all()
    # leaves partition the particles in order
    ls, le = start[leaf], end[leaf]
    assert ls[0] == 0 and le[-1] == n and (ls[1:] == le[:-1]).all()
    keys = a["keys"]
    assert (np.diff(keys.astype(np.float64)) >= 0).all()
    assert sorted(a["perm"].tolist()) == list(range(n))


@pytest.mark.parametrize("dist", ["uniform", "plummer", "dupes", "tiny"])
def test_native_topology_invariants(dist):
    if dist == "uniform":
        p, m = W.uniform_cube(3000, seed=1)
    elif dist == "plummer":
        p, m = W.plummer(5000, seed=2)
    elif dist == "dupes":
        p, m = W.uniform_cube(400, seed=3)
        p = np.concatenate([p, np.repeat(p[:5], 40, axis=0)])
        m = np.full(p.shape[0], 1.0 / p.shape[0], np.float32)
    else:
        p, m = W.uniform_cube(7, seed=4)
    T = O.NativeTree(p, m, leaf_size=16)
    _topology_invariants(T)


def test_native_infinite_beta_is_direct():
    p, m = W.plummer(2000, seed=5)
    T = O.NativeTree(p, m, leaf_size=16)
    T.plan(1e30, 32)
    f, _ = T.force(1e-3)
    want = O.direct_force_soft(p, m, p, 1e-3)
    assert rel_l2(f, want) < 1e-12


@pytest.mark.parametrize("quad,qradius", [(False, 0.0), (True, 0.0), (True, 1.6)])
def test_native_adjoint_matches_finite_differences(quad, qradius):
    rng = np.random.default_rng(6)
    p, m = W.plummer(600, seed=6)
    m = (m * rng.uniform(0.5, 1.5, m.shape)).astype(np.float32)
    w = rng.normal(size=p.shape).astype(np.float32)
    eps = 1e-2
    T = O.NativeTree(p, m, leaf_size=8)
    with O.native_quadrupole_radius(qradius):
        T.plan(2.0, 32)
    if qradius > 0:
        # a mixed plan: some far nodes with the quadrupole, some without
        T0 = O.NativeTree(p, m, leaf_size=8)
        T0.plan(2.0, 32)
        assert 0 < T.quadrupole_interactions() < T0.quadrupole_interactions()
    dx, dm = T.adjoint(w, eps, quad=quad)
    p64 = p.astype(np.float64)
    h = 1e-4
    idx = rng.choice(p.shape[0], 24, replace=False)
    for k in idx:
        for d in range(3):
            pp = p64.copy()
            pp[k, d] += h
            lp = T.force(eps, points=pp.astype(np.float32), masses=m, w=w, quad=quad)[1]
            pp[k, d] -= 2 * h
            lm = T.force(eps, points=pp.astype(np.float32), masses=m, w=w, quad=quad)[1]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - dx[k, d]) <= 2e-3 * (abs(fd) + 1.0), (k, d, fd, dx[k, d])
        mm = m.astype(np.float64).copy()
        dh = 1e-3 * m[k]
        mm[k] += dh
        lp = T.force(eps, points=p, masses=mm.astype(np.float32), w=w, quad=quad)[1]
        mm[k] -= 2 * dh
        lm = T.force(eps, points=p, masses=mm.astype(np.float32), w=w, quad=quad)[1]
        fd = (lp - lm) / (2 * dh)
        assert abs(fd - dm[k]) <= 2e-3 * (abs(fd) + 1.0), (k, fd, dm[k])


def test_native_quadrupole_radius_trades_order_for_accuracy():
    """The quadrupole radius keeps the plan (same far and near lists) and
    only drops the quadrupole of distant nodes: the error sits between the
    monopole's and the full quadrupole's."""
    p, m = W.plummer(20000, seed=9)
    idx = np.random.default_rng(1).choice(p.shape[0], 256, replace=False)
    want = O.direct_force_soft(p, m, p[idx], 1e-3)
    err, counts = {}, {}
    for q in (0.0, 1.6):
        T = O.NativeTree(p, m, leaf_size=16)
        with O.native_quadrupole_radius(q):
            counts[q] = T.plan(2.0, 64)
        err[q] = rel_l2(T.force(1e-3, quad=True)[0][idx], want)
        if q == 0.0:
            err["mono"] = rel_l2(T.force(1e-3, quad=False)[0][idx], want)
            nfar_total = T.quadrupole_interactions()
        else:
            frac = T.quadrupole_interactions() / nfar_total
    assert counts[0.0] == counts[1.6]
    assert 0.2 < frac < 0.8
    assert err[0.0] < err[1.6] < err["mono"]
    assert err[1.6] < 1e-4


def test_native_adjoint_approximates_exact_gradient():
    rng = np.random.default_rng(8)
    p, m = W.plummer(3000, seed=8)
    w = rng.normal(size=p.shape).astype(np.float32)
    T = O.NativeTree(p, m, leaf_size=16)
    T.plan(2.0, 32)
    dx, dm = T.adjoint(w, 1e-3, quad=True)
    ex, em = O.direct_full_adjoint(p, m, w, 1e-3)
    assert rel_l2(dx, ex) < 1e-3
    assert rel_l2(dm, em) < 1e-3


def test_native_linearized_quadrupole_adjoint_matches_finite_differences():
    """With the quadrupole of distant nodes taken to first order about the
    group centre (frozen with the plan), the oracle's adjoint -- the query
    side J w, and per (group, node) dL/dX and dL/dS of W . a_q + V : J --
    equals Richardson-extrapolated central differences of the same frozen
    plan, and agrees with full-loss differences of the evaluator."""
    rng = np.random.default_rng(16)
    p, m = W.plummer(2000, seed=16)
    m = (m * rng.uniform(0.5, 1.5, m.shape)).astype(np.float32)
    w = rng.normal(size=p.shape).astype(np.float32)
    eps = 1e-2
    T = O.NativeTree(p, m, leaf_size=8)
    with O.native_quadrupole_linear(0.5):
        T.plan(2.0, 32)
    lin_target, lin_pairs = T.linear_quadrupole_counts()
    assert 0 < lin_target < T.quadrupole_interactions() and lin_pairs > 0
    dx, dm = T.adjoint(w, eps, quad=True)
    idx = rng.choice(p.shape[0], 30, replace=False)
    fx, fm = T.finite_differences(w, eps, idx, hx=1e-4, hm_rel=1e-4, quad=True)
    fx2, fm2 = T.finite_differences(w, eps, idx, hx=5e-5, hm_rel=5e-5, quad=True)
    assert rel_l2(dx[idx], (4 * fx2 - fx) / 3) < 1e-8
    assert rel_l2(dm[idx], (4 * fm2 - fm) / 3) < 1e-8
    k, h = idx[0], 1e-3
    pp = p.astype(np.float64)
    pp[k, 2] += h
    lp = T.force(eps, points=pp.astype(np.float32), masses=m, w=w, quad=True)[1]
    pp[k, 2] -= 2 * h
    lm = T.force(eps, points=pp.astype(np.float32), masses=m, w=w, quad=True)[1]
    assert abs((lp - lm) / (2 * h) - dx[k, 2]) <= 2e-3 * (abs(dx[k, 2]) + 1.0)


def test_native_winding_number_adjoint_matches_finite_differences():
    """The oracle's winding-number plan (queries in Morton order, groups of 32)
    equals the direct sum in its direct limit, and its adjoint with respect to
    queries, source positions, normals and weights matches central
    differences of the frozen-plan evaluation."""
    p, nrm, m = W.ellipsoid_surface(3000, seed=3)
    rng = np.random.default_rng(1)
    q = rng.uniform(-1.5, 1.5, (200, 3)).astype(np.float32)
    u = rng.normal(size=200).astype(np.float32)
    T = O.NativeTree(p, m, leaf_size=8)
    T.wn_plan(q, 1e30)
    assert np.abs(T.wn_eval(nrm) - O.direct_winding_number(p, nrm, m, q)).max() < 1e-10
    T.wn_plan(q, 2.0)
    dq, dp, dn, dm = T.wn_adjoint(nrm, u)
    p64, n64, q64, m64 = (a.astype(np.float64) for a in (p, nrm, q, m))

    def loss(pp=p64, nn=n64, mm=m64, qq=q64):
        # float64 inputs are rounded to float32 by the evaluator: steps are kept well above that
        return float(np.dot(u, T.wn_eval(nn.astype(np.float32), points=pp.astype(np.float32),
                                         masses=mm.astype(np.float32), queries=qq.astype(np.float32))))

    h = 1e-3
    for i in (3, 50):
        for c in range(3):
            a = q64.copy(); a[i, c] += h; lp = loss(qq=a); a[i, c] -= 2 * h; lm = loss(qq=a)
            assert abs((lp - lm) / (2 * h) - dq[i, c]) <= 2e-3 * (abs(dq[i, c]) + 1e-3)
    for j in (7, 1200):
        a = p64.copy(); a[j, 0] += h; lp = loss(pp=a); a[j, 0] -= 2 * h; lm = loss(pp=a)
        assert abs((lp - lm) / (2 * h) - dp[j, 0]) <= 2e-3 * (abs(dp[j, 0]) + 1e-3)
        a = n64.copy(); a[j, 1] += h; lp = loss(nn=a); a[j, 1] -= 2 * h; lm = loss(nn=a)
        assert abs((lp - lm) / (2 * h) - dn[j, 1]) <= 2e-3 * (abs(dn[j, 1]) + 1e-3)
        a = m64.copy(); hm = 1e-2 * m64[j]; a[j] += hm; lp = loss(mm=a); a[j] -= 2 * hm; lm = loss(mm=a)
        assert abs((lp - lm) / (2 * hm) - dm[j]) <= 2e-3 * (abs(dm[j]) + 1e-3)


def test_stochastic_restatement_unbiased_and_accurate():
    """The stochastic estimator's restatement on the oracle's own tree: the
    mean over seeds converges to its expectation (the group walk at beta =
    2), which meets the FP64 direct sum; 32 drawn nodes per query stay
    within the error the coarse opening leaves to sample."""
    n = 6000
    p, m = W.plummer(n, seed=8)
    T = O.NativeTree(p, m, leaf_size=16)
    rec = T.node_records()
    sp, perm = T.sorted_sources()
    runs, ex = [], None
    for s in range(24):
        est, e, walks = O.native_stochastic(sp, perm, rec, beta_coarse=1.0, samples=4, seed=s, expectation=ex is None)
        ex = e if ex is None else ex
        assert walks > 0
        runs.append(est)
    runs = np.stack(runs)
    err_one = rel_l2(runs[0], ex)
    err_mean = rel_l2(runs.mean(0), ex)
    assert err_mean < 0.35 * err_one  # ~1 / sqrt(24) = 0.2 for an unbiased estimator
    idx = np.arange(0, n, 7)
    ref = O.direct_force_soft(p, m, p[idx], 1e-3)
    assert rel_l2(ex[idx], ref) < 1e-4
    est, _, _ = O.native_stochastic(sp, perm, rec, beta_coarse=1.0, samples=32, seed=1, expectation=False)
    assert rel_l2(est[idx], ref) < 2e-3


def test_stochastic_plan_adjoint_matches_finite_differences():
    """The stochastic estimate as a frozen plan with per-term coefficients
    (orc_native_stochastic_plan): its value equals the restatement's
    estimate, and its adjoint (the VJP with the draws held fixed) matches
    FP64 central differences of the same frozen plan, for positions and
    masses."""
    n = 3000
    p, m = W.plummer(n, seed=9)
    T = O.NativeTree(p, m, leaf_size=16)
    rec = T.node_records()
    sp, perm = T.sorted_sources()
    est, _, _ = O.native_stochastic(sp, perm, rec, beta_coarse=1.0, samples=8, seed=4, expectation=False)
    assert T.stochastic_plan(rec, beta_coarse=1.0, samples=8, seed=4) > 0
    val, _ = T.force(1e-3, quad=True)
    # the plan sums the same terms with the double moments instead of the float records
    assert rel_l2(val, est) < 1e-5
    w = np.random.default_rng(10).normal(size=(n, 3)).astype(np.float32)
    dx, dm = T.adjoint(w, 1e-3, quad=True)
    idx = np.random.default_rng(11).choice(n, 40, replace=False)
    fx1, fm1 = T.finite_differences(w, 1e-3, idx, hx=1e-4, hm_rel=1e-4, quad=True)
    fx2, fm2 = T.finite_differences(w, 1e-3, idx, hx=5e-5, hm_rel=5e-5, quad=True)
    fx, fm = (4 * fx2 - fx1) / 3, (4 * fm2 - fm1) / 3  # Richardson
    assert rel_l2(dx[idx], fx) < 1e-5
    assert rel_l2(dm[idx], fm) < 1e-5
