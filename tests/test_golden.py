"""CPU tests: the oracle pinned to golden fixtures produced by the
reference's own GPU plugin (src/sbh_ffi.cu, unmodified, compiled into
oracle/_ref and run on a B200 by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import sbh_oracle as O
from conftest import rel_l2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} missing")
    return np.load(path)


def test_direct_fixture():
    g = _load("direct_reference.npz")
    got = O.direct_force_soft(g["points"], g["masses"], g["queries"], 5e-2, 0.9)
    np.testing.assert_allclose(got, g["force"], rtol=5e-5, atol=5e-6)
    got = O.direct_force_soft_vjp(g["points"], g["masses"], g["queries"], g["cot"], 7e-2, 1.4)
    np.testing.assert_allclose(got, g["vjp"], rtol=1e-4, atol=1e-5)
    for dim in (2, 3):
        got = O.bruteforce_gravity(g[f"bf{dim}_points"], g[f"bf{dim}_masses"], g[f"bf{dim}_queries"])
        np.testing.assert_allclose(got, g[f"bf{dim}_out"], rtol=2e-5)


def _fields(node):
    a = node.reshape(-1, 104)
    u = a[:, :48].copy().view(np.uint32)
    return dict(start=u[:, 0], end=u[:, 1], parent=u[:, 2], first=u[:, 3], child=u[:, 4:12], mask=a[:, 48],
                depth=a[:, 49], leaf=a[:, 50], geom=a[:, 52:72].copy().view(np.float32),
                contrib=a[:, 72:104].copy().view(np.float32))


@pytest.mark.parametrize("case", ["uniform_d3", "uniform_d5", "plummer_d3", "plummer_d5"])
def test_octree8_build_fixture(case):
    g = _load("octree8_reference.npz")
    leaf, node, contrib, codes, perm = O.build_octree8(g[case + "_points"], g[case + "_normals"], g[case + "_masses"],
                                                       g[case + "_min"], g[case + "_max"], int(case[-1]))
    a, b = _fields(node), _fields(g[case + "_node"])
    # integer topology: identical except where the reference's approximate
    # division puts a point on the other side of a cell wall
    bad = int((a["start"] != b["start"]).sum() + (a["end"] != b["end"]).sum())
    assert bad <= 4, bad
    for k in ("parent", "first", "child", "depth"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    np.testing.assert_array_equal(a["geom"], b["geom"])
    if bad == 0:
        np.testing.assert_array_equal(a["mask"], b["mask"])
        np.testing.assert_allclose(a["contrib"], b["contrib"], rtol=5e-5, atol=1e-6)
        la = leaf.reshape(-1, 32).copy().view(np.float32)
        lb = g[case + "_leaf"].reshape(-1, 32).copy().view(np.float32)
        for s, e, lf in zip(b["start"], b["end"], b["leaf"]):
            if lf and e > s:
                assert sorted(map(tuple, la[s:e])) == sorted(map(tuple, lb[s:e]))
    np.testing.assert_array_equal(contrib.reshape(-1, 32), node.reshape(-1, 104)[:, 72:])


@pytest.mark.parametrize("case", ["uniform_d5", "plummer_d5"])
def test_octree8_traversal_fixture(case):
    g = _load("octree8_reference.npz")
    leaf, node, q, cot = g[case + "_leaf"], g[case + "_node"], g[case + "_queries"], g[case + "_cot"]
    got, _ = O.bh_octree8(leaf, node, q, 2.0, O.KERNEL_GRAV_GRAD)
    assert rel_l2(got, g[case + "_bh_beta2"]) < 1e-5
    for tag, (eps, cut, prune, mult) in {"soft": (5e-2, 1.5, False, 4.0), "softprune": (5e-2, 0.3, True, 2.0),
                                         "plummer": (1e-3, 1e6, True, 4.0)}.items():
        got, _ = O.bh_octree8(leaf, node, q, 2.0, O.KERNEL_SOFT, eps=eps, cutoff=cut, prune_enabled=prune,
                              prune_r_cut_mult=mult)
        assert rel_l2(got, g[case + f"_{tag}"]) < 1e-5, tag
        got, _ = O.bh_octree8(leaf, node, q, 2.0, O.KERNEL_SOFT_VJP, eps=eps, cutoff=cut, prune_enabled=prune,
                              prune_r_cut_mult=mult, cot=cot)
        assert rel_l2(got, g[case + f"_{tag}_vjp"]) < 1e-5, tag


def test_octree8_periodic_fixture():
    g = _load("octree8_reference.npz")
    got, _ = O.bh_octree8(g["periodic_leaf"], g["periodic_node"], g["periodic_points"][:32], 1.8,
                          O.KERNEL_GRAV_GRAD, periodic=True, box=2.0)
    assert rel_l2(got, g["periodic_force"]) < 1e-5
