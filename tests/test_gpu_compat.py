"""GPU parity of the reference-layout ("compat") entry points.

Each test runs the library's CUDA path through the C ABI (via sbh_b200) and
compares it with
  * the reference's own kernels (src/sbh_ffi.cu compiled into
    oracle/_ref/libsbh_ref_gpu.so) on the SAME inputs and buffers, and
  * the CPU oracle (oracle/sbh_oracle.c), which evaluates the same algorithm
    with float decisions and double sums.
Tolerances: integer/byte fields bit-exact; float sums within 1e-5 relative
L2 (the classic-BH parity tolerance against the reference's kernels) unless
stated otherwise.
"""
import numpy as np
import pytest
import torch

import sbh_b200 as B
import sbh_oracle as O
import sbh_workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu

HAVE_REF = O.available("libsbh_ref_gpu.so")
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="reference GPU build missing (make -C oracle ref)")


def _t(a, dev, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), device=dev, dtype=dtype)


def _S():
    return torch.cuda.current_stream().cuda_stream


def ref_build_octree8(dev, p, nrm, m, mn, mx, depth):
    L = O.refgpu()
    n = p.shape[0]
    total = O.octree8_total_nodes(depth)
    leaf = torch.zeros(n * 32, dtype=torch.uint8, device=dev)
    node = torch.zeros(total * 104, dtype=torch.uint8, device=dev)
    contrib = torch.zeros(total * 32, dtype=torch.uint8, device=dev)
    P, N, M, MN, MX = _t(p, dev), _t(nrm, dev), _t(m, dev), _t(mn, dev), _t(mx, dev)
    O.refgpu_check(L.ref_build_octree8(_S(), P.data_ptr(), N.data_ptr(), M.data_ptr(), n, MN.data_ptr(),
                                       MX.data_ptr(), leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                       contrib.data_ptr(), contrib.numel(), depth))
    torch.cuda.synchronize()
    return leaf, node, contrib


def node_fields(node_bytes):
    a = np.asarray(node_bytes.cpu() if isinstance(node_bytes, torch.Tensor) else node_bytes).reshape(-1, 104)
    u = a[:, :48].copy().view(np.uint32)
    f = a[:, 52:72].copy().view(np.float32)
    c = a[:, 72:104].copy().view(np.float32)
    return dict(start=u[:, 0], end=u[:, 1], parent=u[:, 2], first_child=u[:, 3], child=u[:, 4:12],
                mask=a[:, 48], depth=a[:, 49], is_leaf=a[:, 50], geom=f, contrib=c)


def leaf_records(leaf_bytes):
    a = np.asarray(leaf_bytes.cpu() if isinstance(leaf_bytes, torch.Tensor) else leaf_bytes)
    return a.reshape(-1, 32).copy().view(np.float32)


def assert_same_octree8(mine, ref, exact_geom=True):
    """Topology bit-exact, per-cell particle multisets equal, sums close."""
    a, b = node_fields(mine), node_fields(ref)
    for k in ("start", "end", "parent", "first_child", "child", "mask", "depth", "is_leaf"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    if exact_geom:
        np.testing.assert_array_equal(a["geom"], b["geom"])
    else:
        np.testing.assert_allclose(a["geom"], b["geom"], rtol=1e-6)
    np.testing.assert_allclose(a["contrib"], b["contrib"], rtol=2e-5, atol=1e-6)
    return a


def assert_same_leaves(leaf_a, leaf_b, starts, ends, is_leaf):
    la, lb = leaf_records(leaf_a), leaf_records(leaf_b)
    assert la.shape == lb.shape
    for s, e, lf in zip(starts, ends, is_leaf):
        if lf and e > s:
            ka = sorted(map(tuple, la[s:e]))
            kb = sorted(map(tuple, lb[s:e]))
            assert ka == kb


# --------------------------------------------------------------------------
# direct sums (reference tests test_jax_ffi_tree_builder.py:20-123)
# --------------------------------------------------------------------------
def test_softened_direct_force_matches_oracle_and_reference(cuda):
    rng = np.random.default_rng(23)
    p = rng.uniform(-1, 1, (96, 3)).astype(np.float32)
    m = rng.uniform(0.1, 1.3, 96).astype(np.float32)
    q = rng.uniform(-0.7, 0.7, (31, 3)).astype(np.float32)
    got = B.softened_direct_force(p, m, q, softening_scale=5e-2, cutoff_scale=0.9).cpu().numpy()
    want = O.direct_force_soft(p, m, q, 5e-2, 0.9)
    np.testing.assert_allclose(got, want, rtol=5e-5, atol=5e-6)
    if HAVE_REF:
        out = torch.zeros((31, 3), device=cuda)
        P, M, Q = _t(p, cuda), _t(m, cuda), _t(q, cuda)
        O.refgpu_check(O.refgpu().ref_direct_force_soft(_S(), P.data_ptr(), M.data_ptr(), 96, Q.data_ptr(), 31,
                                                        out.data_ptr(), 5e-2, 0.9, 0, 1.0, 256))
        np.testing.assert_allclose(got, out.cpu().numpy(), rtol=5e-5, atol=5e-6)


def test_softened_direct_force_vjp_matches_oracle(cuda):
    rng = np.random.default_rng(31)
    p = rng.uniform(-1, 1, (64, 3)).astype(np.float32)
    m = rng.uniform(0.2, 1.1, 64).astype(np.float32)
    q = rng.uniform(-0.5, 0.5, (17, 3)).astype(np.float32)
    g = rng.normal(size=(17, 3)).astype(np.float32)
    got = B.softened_direct_force_vjp(p, m, q, g, softening_scale=7e-2, cutoff_scale=1.4).cpu().numpy()
    want = O.direct_force_soft_vjp(p, m, q, g, 7e-2, 1.4)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-5)


def test_recompute_vjp_equals_explicit_query_side_vjp(cuda):
    rng = np.random.default_rng(41)
    p = torch.tensor(rng.uniform(-1, 1, (72, 3)), dtype=torch.float32, device=cuda, requires_grad=True)
    m = torch.tensor(rng.uniform(0.2, 1.1, 72), dtype=torch.float32, device=cuda, requires_grad=True)
    cot = torch.tensor(rng.normal(size=(72, 3)), dtype=torch.float32, device=cuda)
    f = B.softened_direct_force_recompute_vjp(p, m, softening_scale=6e-2, cutoff_scale=1.1)
    (f * cot).sum().backward()
    want = B.softened_direct_force_vjp(p.detach(), m.detach(), p.detach(), cot, softening_scale=6e-2, cutoff_scale=1.1)
    np.testing.assert_allclose(p.grad.cpu().numpy(), want.cpu().numpy(), rtol=1e-6, atol=1e-6)
    assert float(m.grad.abs().max()) == 0.0


def test_direct_force_large_against_fp64_oracle(cuda):
    p, m = W.plummer(20000, seed=3)
    q = p[::37]
    got = B.softened_direct_force(p, m, q, softening_scale=1e-3, cutoff_scale=1e6).cpu().numpy()
    want = O.direct_force_soft(p, m, q, 1e-3, 1e6)
    assert rel_l2(got, want) < 2e-6


def test_bruteforce_gravity_2d_3d(cuda):
    rng = np.random.default_rng(5)
    for dim in (2, 3):
        p = rng.uniform(-1, 1, (500, dim)).astype(np.float32)
        m = rng.uniform(0.1, 1, 500).astype(np.float32)
        q = rng.uniform(-1, 1, (100, dim)).astype(np.float32)
        got = B.brute_force_gravity(p, m, q).cpu().numpy()
        np.testing.assert_allclose(got, O.bruteforce_gravity(p, m, q), rtol=1e-5)


# --------------------------------------------------------------------------
# octree8 build (src/sbh_ffi.cu:1039-1420)
# --------------------------------------------------------------------------
@pytest.mark.parametrize("dist,depth", [("uniform", 3), ("uniform", 5), ("plummer", 5), ("plummer", 7)])
def test_octree8_build_matches_oracle(cuda, dist, depth):
    p, m = W.uniform_cube(4000, seed=2) if dist == "uniform" else W.plummer(4000, seed=2)
    nrm = np.random.default_rng(3).normal(size=p.shape).astype(np.float32)
    mn = p.min(0) - np.float32(1e-3)
    mx = p.max(0) + np.float32(1e-3)
    leaf, node, contrib = B.build_octree8_buffers_with_contrib(p, nrm, m, mn, mx, max_depth=depth)
    oleaf, onode, ocontrib, codes, perm = O.build_octree8(p, nrm, m, mn, mx, depth)
    # The oracle divides exactly, the reference's flags divide approximately:
    # a point within an ulp of a cell wall may land in the neighbour cell.
    a, b = node_fields(node), node_fields(onode)
    mismatch = int((a["start"] != b["start"]).sum())
    assert mismatch <= 2 * depth, f"{mismatch} node starts differ from the IEEE oracle"
    if mismatch == 0:
        np.testing.assert_array_equal(leaf.cpu().numpy(), oleaf)  # same stable order
        np.testing.assert_allclose(a["contrib"], b["contrib"], rtol=1e-6, atol=1e-7)
    np.testing.assert_array_equal(a["geom"], b["geom"])
    np.testing.assert_array_equal(contrib.cpu().numpy().reshape(-1, 32), node.cpu().numpy().reshape(-1, 104)[:, 72:])


@needs_ref
@pytest.mark.parametrize("dist,depth", [("uniform", 4), ("plummer", 6)])
def test_octree8_build_matches_reference(cuda, dist, depth):
    p, m = W.uniform_cube(5000, seed=8) if dist == "uniform" else W.plummer(5000, seed=8)
    nrm = np.random.default_rng(4).normal(size=p.shape).astype(np.float32)
    mn = p.min(0) - np.float32(1e-3)
    mx = p.max(0) + np.float32(1e-3)
    leaf, node, _ = B.build_octree8_buffers_with_contrib(p, nrm, m, mn, mx, max_depth=depth)
    rleaf, rnode, _ = ref_build_octree8(cuda, p, nrm, m, mn, mx, depth)
    f = assert_same_octree8(node, rnode)
    assert_same_leaves(leaf, rleaf, f["start"], f["end"], f["is_leaf"])


def test_octree8_build_rejects_bad_arguments(cuda):
    p, m = W.uniform_cube(100, seed=1)
    with pytest.raises(ValueError):
        B.build_octree8_buffers(p, np.zeros_like(p), m, max_depth=0)
    with pytest.raises(ValueError):
        B.build_octree8_buffers(p, np.zeros_like(p), m, max_depth=11)
    with pytest.raises(ValueError):  # zero span: detected on the device
        B.build_octree8_buffers(p, np.zeros_like(p), m, np.ones(3, np.float32), np.ones(3, np.float32), max_depth=3)


def test_octree8_build_empty_input(cuda):
    p = np.zeros((0, 3), np.float32)
    leaf, node, contrib = B.build_octree8_buffers_with_contrib(p, p, np.zeros(0, np.float32), np.zeros(3, np.float32),
                                                               np.ones(3, np.float32), max_depth=2)
    f = node_fields(node)
    assert leaf.numel() == 0
    assert (f["start"] == 0).all() and (f["end"] == 0).all() and (f["contrib"][:, 6] == 0).all()


# --------------------------------------------------------------------------
# octree8 traversals (src/sbh_ffi.cu:1950-2144)
# --------------------------------------------------------------------------
def _build_both(cuda, n=3000, depth=5, seed=5, scale=0.3):
    p, m = W.plummer(n, seed=seed)
    p = p * np.float32(scale)
    nrm = np.zeros_like(p)
    mn = p.min(0) - np.float32(1e-3)
    mx = p.max(0) + np.float32(1e-3)
    leaf, node = B.build_octree8_buffers(p, nrm, m, mn, mx, max_depth=depth)
    return p, m, leaf, node


@pytest.mark.parametrize("kind", ["grav", "soft", "softprune", "plummer"])
def test_octree8_traversal_matches_oracle(cuda, kind):
    p, m, leaf, node = _build_both(cuda)
    rng = np.random.default_rng(9)
    q = np.concatenate([p[:500], rng.uniform(p.min(0), p.max(0), (100, 3)).astype(np.float32)])
    cot = rng.normal(size=q.shape).astype(np.float32)
    lb, nb = leaf.cpu().numpy(), node.cpu().numpy()
    if kind == "grav":
        got = B.barnes_hut_force_octree8(leaf, node, q, beta=2.0, check_status=True).cpu().numpy()
        want, _ = O.bh_octree8(lb, nb, q, 2.0, O.KERNEL_GRAV_GRAD)
        assert rel_l2(got, want) < 1e-5
        return
    eps, cut, prune, mult = {"soft": (5e-2, 1.5, False, 4.0), "softprune": (5e-2, 0.3, True, 2.0),
                             "plummer": (1e-3, 1e6, True, 4.0)}[kind]
    got = B.softened_barnes_hut_force_octree8(leaf, node, q, beta=2.0, softening_scale=eps, cutoff_scale=cut,
                                              prune_enabled=prune, prune_r_cut_mult=mult, check_status=True)
    want, _ = O.bh_octree8(lb, nb, q, 2.0, O.KERNEL_SOFT, eps=eps, cutoff=cut, prune_enabled=prune,
                           prune_r_cut_mult=mult)
    assert rel_l2(got.cpu().numpy(), want) < 1e-5
    gv = B.softened_barnes_hut_force_octree8_vjp(leaf, node, q, cot, beta=2.0, softening_scale=eps, cutoff_scale=cut,
                                                 prune_enabled=prune, prune_r_cut_mult=mult, check_status=True)
    wv, _ = O.bh_octree8(lb, nb, q, 2.0, O.KERNEL_SOFT_VJP, eps=eps, cutoff=cut, prune_enabled=prune,
                         prune_r_cut_mult=mult, cot=cot)
    assert rel_l2(gv.cpu().numpy(), wv) < 1e-5


@needs_ref
def test_octree8_traversals_match_reference_kernels_on_same_buffers(cuda):
    p, m, leaf, node = _build_both(cuda, n=4000, depth=6)
    rng = np.random.default_rng(12)
    q = np.concatenate([p[:700], rng.uniform(p.min(0), p.max(0), (100, 3)).astype(np.float32)])
    cot = rng.normal(size=q.shape).astype(np.float32)
    L = O.refgpu()
    Q, C = _t(q, cuda), _t(cot, cuda)
    nq = q.shape[0]

    def ref(fn, args):
        out = torch.zeros((nq, 3), device=cuda)
        O.refgpu_check(fn(_S(), *args(out)))
        torch.cuda.synchronize()
        return out.cpu().numpy()

    lp, lb, np_, nb = leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel()
    r = ref(L.ref_bh_force_octree8, lambda o: (lp, lb, np_, nb, Q.data_ptr(), nq, o.data_ptr(), 2.0, 0, 1.0, 256))
    assert rel_l2(B.barnes_hut_force_octree8(leaf, node, q, beta=2.0).cpu().numpy(), r) < 1e-5
    for eps, cut, prune, mult in ((5e-2, 1.5, 0, 4.0), (5e-2, 0.3, 1, 2.0)):
        r = ref(L.ref_bh_force_octree8_soft, lambda o: (lp, lb, np_, nb, Q.data_ptr(), nq, o.data_ptr(), 2.0, eps, cut,
                                                        prune, mult, 0, 1.0, 256))
        got = B.softened_barnes_hut_force_octree8(leaf, node, q, beta=2.0, softening_scale=eps, cutoff_scale=cut,
                                                  prune_enabled=bool(prune), prune_r_cut_mult=mult)
        assert rel_l2(got.cpu().numpy(), r) < 1e-5
        r = ref(L.ref_bh_force_octree8_soft_vjp, lambda o: (lp, lb, np_, nb, Q.data_ptr(), nq, C.data_ptr(),
                                                            o.data_ptr(), 2.0, eps, cut, prune, mult, 0, 1.0, 256))
        got = B.softened_barnes_hut_force_octree8_vjp(leaf, node, q, cot, beta=2.0, softening_scale=eps,
                                                      cutoff_scale=cut, prune_enabled=bool(prune),
                                                      prune_r_cut_mult=mult)
        assert rel_l2(got.cpu().numpy(), r) < 1e-5


@needs_ref
@pytest.mark.parametrize("soft", [0, 1])
@pytest.mark.parametrize("vjp", [False, True])
@pytest.mark.parametrize("n,depth,nq", [(3000, 5, 600), (30000, 6, 20000)])
def test_stochastic_octree8_fixed_seed_matches_reference(cuda, soft, vjp, n, depth, nq):
    p, m, leaf, node = _build_both(cuda, n=n, depth=depth)
    rng = np.random.default_rng(13)
    q = p[:nq]
    cot = rng.normal(size=q.shape).astype(np.float32)
    L = O.refgpu()
    Q, C = _t(q, cuda), _t(cot, cuda)
    nq = q.shape[0]
    out = torch.zeros((nq, 3), device=cuda)
    lp, lb, np_, nb = leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel()
    if vjp:
        O.refgpu_check(L.ref_stochastic_bh_force_octree8_vjp(_S(), soft, lp, lb, np_, nb, Q.data_ptr(), nq,
                                                             C.data_ptr(), out.data_ptr(), 2, 7, 1.0, 5e-2, 1.5, 1,
                                                             4.0, 0, 1.0, 256))
        fn = B.softened_stochastic_barnes_hut_force_octree8_vjp if soft else B.stochastic_barnes_hut_force_octree8_vjp
        kw = dict(softening_scale=5e-2, cutoff_scale=1.5) if soft else {}
        got = fn(leaf, node, q, cot, samples_per_subdomain=2, seed=7, beta=1.0, **kw)
    else:
        O.refgpu_check(L.ref_stochastic_bh_force_octree8(_S(), soft, lp, lb, np_, nb, Q.data_ptr(), nq,
                                                         out.data_ptr(), 2, 7, 1.0, 5e-2, 1.5, 1, 4.0, 0, 1.0, 256))
        fn = B.softened_stochastic_barnes_hut_force_octree8 if soft else B.stochastic_barnes_hut_force_octree8
        kw = dict(softening_scale=5e-2, cutoff_scale=1.5) if soft else {}
        got = fn(leaf, node, q, samples_per_subdomain=2, seed=7, beta=1.0, **kw)
    torch.cuda.synchronize()
    r = out.cpu().numpy()
    g = got.cpu().numpy()
    row = np.linalg.norm(g - r, axis=1) / np.maximum(np.linalg.norm(r, axis=1), 1e-30)
    # Same curand streams and buffers, and the same opening probabilities:
    # every row takes the reference's sampled paths, so no row may differ by
    # more than the summation order of its terms explains (largest seen over
    # the 2 x 4 cases: 1.0e-5 on one row of 20,000). A flipped Russian-roulette
    # decision would show as an O(1) row error.
    assert row.max() < 1e-4, f"{int((row >= 1e-4).sum())} rows differ, worst {row.max():.2e}"


def test_stochastic_same_seed_same_result_and_prune_noop(cuda):
    # test_jax_ffi_tree_builder.py:415-469 with this library
    box = 2.0
    rng = np.random.default_rng(11)
    p = rng.uniform(0, box, (320, 3)).astype(np.float32)
    m = np.ones(320, np.float32)
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, np.zeros(3, np.float32),
                                         np.full(3, box, np.float32), max_depth=5)
    q = p[:64]
    kw = dict(samples_per_subdomain=2, seed=5, softening_scale=5e-2, cutoff_scale=0.4)
    a = B.softened_stochastic_barnes_hut_force_octree8(leaf, node, q, prune_enabled=False, **kw)
    b = B.softened_stochastic_barnes_hut_force_octree8(leaf, node, q, prune_enabled=True, prune_r_cut_mult=1e6, **kw)
    c = B.softened_stochastic_barnes_hut_force_octree8(leaf, node, q, prune_enabled=False, **kw)
    np.testing.assert_allclose(a.cpu().numpy(), b.cpu().numpy(), rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(a.cpu().numpy(), c.cpu().numpy())


def test_octree8_periodic_shift_invariance(cuda):
    # test_jax_ffi_tree_builder.py:264-305
    box = 2.0
    rng = np.random.default_rng(3)
    p = rng.uniform(0, box, (192, 3)).astype(np.float32)
    m = np.ones(192, np.float32)
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, np.zeros(3, np.float32),
                                         np.full(3, box, np.float32), max_depth=5)
    q = p[:32]
    qs = q + np.array([box, 0, 0], np.float32)
    f0 = B.barnes_hut_force_octree8(leaf, node, q, beta=1.8, periodic=True, box_length=box).cpu().numpy()
    f1 = B.barnes_hut_force_octree8(leaf, node, qs, beta=1.8, periodic=True, box_length=box).cpu().numpy()
    np.testing.assert_allclose(f0, f1, rtol=1e-2, atol=5e-3)
    s0 = B.softened_barnes_hut_force_octree8(leaf, node, q, beta=1.8, softening_scale=5e-2, cutoff_scale=0.3,
                                             prune_enabled=True, prune_r_cut_mult=3.0, periodic=True,
                                             box_length=box).cpu().numpy()
    s1 = B.softened_barnes_hut_force_octree8(leaf, node, qs, beta=1.8, softening_scale=5e-2, cutoff_scale=0.3,
                                             prune_enabled=True, prune_r_cut_mult=3.0, periodic=True,
                                             box_length=box).cpu().numpy()
    np.testing.assert_allclose(s0, s1, rtol=1e-2, atol=5e-3)


def test_octree8_prune_large_cutoff_matches_disabled(cuda):
    # test_jax_ffi_tree_builder.py:308-360
    box = 2.0
    rng = np.random.default_rng(11)
    p = rng.uniform(0, box, (320, 3)).astype(np.float32)
    m = np.ones(320, np.float32)
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, np.zeros(3, np.float32),
                                         np.full(3, box, np.float32), max_depth=5)
    a = B.softened_barnes_hut_force_octree8(leaf, node, p, softening_scale=5e-2, cutoff_scale=0.4,
                                            prune_enabled=False).cpu().numpy()
    b = B.softened_barnes_hut_force_octree8(leaf, node, p, softening_scale=5e-2, cutoff_scale=0.4, prune_enabled=True,
                                            prune_r_cut_mult=1e6).cpu().numpy()
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6)


def test_octree8_recompute_vjp_matches_fixed_tree_vjp(cuda):
    # test_jax_custom_vjp_recompute.py:415-461
    rng = np.random.default_rng(104)
    p = torch.tensor(rng.uniform(-1, 1, (104, 3)), dtype=torch.float32, device=cuda, requires_grad=True)
    m = torch.tensor(rng.uniform(0.5, 1.5, 104), dtype=torch.float32, device=cuda)
    cot = torch.tensor(rng.normal(size=(104, 3)), dtype=torch.float32, device=cuda)
    kw = dict(beta=2.0, softening_scale=5e-2, cutoff_scale=1.2)
    f = B.softened_barnes_hut_force_octree8_recompute_vjp(p, m, max_depth=6, **kw)
    (f * cot).sum().backward()
    leaf, node = B.build_octree8_buffers(p.detach(), torch.zeros_like(p), m, max_depth=6)
    want = B.softened_barnes_hut_force_octree8_vjp(leaf, node, p.detach(), cot, **kw)
    np.testing.assert_allclose(p.grad.cpu().numpy(), want.cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_octree8_large_build_and_force_sanity(cuda):
    """N = 262,144 Plummer at depth 7: mass conservation, permutation and force vs FP64 direct on a subset."""
    n = 262144
    p, m = W.plummer(n, seed=21)
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, max_depth=7)
    f = node_fields(node)
    assert f["end"][0] == n and abs(float(f["contrib"][0, 6]) - 1.0) < 1e-5
    lr = leaf_records(leaf)
    assert np.isclose(lr[:, 6].sum(dtype=np.float64), 1.0, rtol=1e-6)
    q = p[::257]
    got = B.softened_barnes_hut_force_octree8(leaf, node, q, beta=2.0, softening_scale=1e-3, cutoff_scale=1e6,
                                              check_status=True).cpu().numpy()
    want = O.direct_force_soft(p, m, q, 1e-3, 1e6)
    assert rel_l2(got, want) < 5e-3  # octree8's geometric-centre criterion (reference README: ~1e-2)


def test_octree8_block_size_changes_no_result(cuda):
    """The warp-cooperative traversal with 1 to 32 warps per block (the
    caller's `threads`) gives the same rows bit for bit, and so does the
    one-thread-per-query kernel (a workspace without room for the order);
    the autotuner picks one of its candidates."""
    p, m = W.plummer(30000, seed=43)
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, p.min(0) - 1e-3, p.max(0) + 1e-3, max_depth=6)
    q = p[:20000]
    kw = dict(beta=2.0, softening_scale=1e-2, cutoff_scale=0.5, prune_enabled=True, prune_r_cut_mult=4.0)
    outs = [B.softened_barnes_hut_force_octree8(leaf, node, q, threads=th, **kw) for th in (32, 96, 256, 1024)]
    torch.cuda.synchronize()
    for o in outs[1:]:
        assert torch.equal(outs[0], o)
    L = B.lib()
    Q = torch.tensor(q, device=cuda)
    ws = torch.empty(int(L.sbh_traversal_workspace_bytes()), dtype=torch.uint8, device=cuda)
    out = torch.empty_like(Q)
    assert L.sbh_barnes_hut_force_octree8_soft(torch.cuda.current_stream(cuda).cuda_stream, leaf.data_ptr(),
                                               leaf.numel(), node.data_ptr(), node.numel(), Q.data_ptr(), Q.shape[0],
                                               out.data_ptr(), 2.0, 1e-2, 0.5, 1, 4.0, 0, 1.0, 256, ws.data_ptr(),
                                               ws.numel()) == 0
    torch.cuda.synchronize()
    assert torch.equal(outs[0], out)
    tuned = B.autotune_octree8(leaf, node, q, **kw)
    assert tuned["threads"] in B.AUTOTUNE_OCTREE8_THREADS and len(tuned["trials"]) == 4


def test_octree8_query_order_changes_no_result(cuda):
    """With the ordered workspace the per-query octree8 traversals take the
    queries in Morton order; every output row must equal the input-order
    run bit for bit (classic, softened with prune, both VJPs, stochastic and
    its VJP)."""
    p, m = W.plummer(30000, seed=41)
    nrm = np.zeros_like(p)
    leaf, node = B.build_octree8_buffers(p, nrm, m, p.min(0) - 1e-3, p.max(0) + 1e-3, max_depth=6)
    rng = np.random.default_rng(42)
    q = p[rng.permutation(p.shape[0])[:20000]]
    cot = rng.normal(size=q.shape).astype(np.float32)
    Q, C = torch.tensor(q, device=cuda), torch.tensor(cot, device=cuda)
    nq = q.shape[0]
    L = B.lib()
    big = torch.empty(int(L.sbh_traversal_ordered_workspace_bytes(nq)), dtype=torch.uint8, device=cuda)
    small = torch.empty(int(L.sbh_traversal_workspace_bytes()), dtype=torch.uint8, device=cuda)
    s = torch.cuda.current_stream(cuda).cuda_stream
    lp, lb, np_, nb = leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel()

    def both(call):
        outs = []
        for ws in (big, small):
            out = torch.full((nq, 3), float("nan"), device=cuda)
            assert call(out.data_ptr(), ws.data_ptr(), ws.numel()) == 0, B.last_error()
            outs.append(out)
        torch.cuda.synchronize()
        assert torch.equal(outs[0], outs[1])
        return outs[0]

    both(lambda o, w, wb: L.sbh_barnes_hut_force_octree8(s, lp, lb, np_, nb, Q.data_ptr(), nq, o, 2.0, 0, 1.0, 256,
                                                         w, wb))
    both(lambda o, w, wb: L.sbh_barnes_hut_force_octree8_vjp(s, lp, lb, np_, nb, Q.data_ptr(), nq, C.data_ptr(), o,
                                                             2.0, 0, 1.0, 256, w, wb))
    both(lambda o, w, wb: L.sbh_barnes_hut_force_octree8_soft(s, lp, lb, np_, nb, Q.data_ptr(), nq, o, 2.0, 1e-2, 0.5,
                                                              1, 4.0, 0, 1.0, 256, w, wb))
    both(lambda o, w, wb: L.sbh_barnes_hut_force_octree8_soft_vjp(s, lp, lb, np_, nb, Q.data_ptr(), nq, C.data_ptr(),
                                                                  o, 2.0, 1e-2, 0.5, 1, 4.0, 0, 1.0, 256, w, wb))
    # The attenuation range against the depth-6 leaf cells (about 0.3 wide):
    # no pair attenuated (the "no cutoff" convention of 1e6 box sizes); an
    # att = 1 radius of cutoff / 256 = 0.5, which some leaves lie wholly
    # inside and others straddle; and a periodic box (scalar pair form).
    span = float((p.max(0) - p.min(0)).max())
    for cut, per, box in ((1e6 * span, 0, 1.0), (128.0, 0, 1.0), (0.5, 1, 1.1 * span)):
        both(lambda o, w, wb: L.sbh_barnes_hut_force_octree8_soft(s, lp, lb, np_, nb, Q.data_ptr(), nq, o, 2.0, 1e-2,
                                                                  cut, 0, 4.0, per, box, 256, w, wb))
        both(lambda o, w, wb: L.sbh_barnes_hut_force_octree8_soft_vjp(s, lp, lb, np_, nb, Q.data_ptr(), nq,
                                                                      C.data_ptr(), o, 2.0, 1e-2, cut, 0, 4.0, per,
                                                                      box, 256, w, wb))
    for soft in (0, 1):
        both(lambda o, w, wb: L.sbh_stochastic_bh_force_octree8(s, soft, lp, lb, np_, nb, Q.data_ptr(), nq, o, 2, 7,
                                                                2.0, 1e-2, 0.5, 1, 4.0, 0, 1.0, 256, w, wb))
        both(lambda o, w, wb: L.sbh_stochastic_bh_force_octree8_vjp(s, soft, lp, lb, np_, nb, Q.data_ptr(), nq,
                                                                    C.data_ptr(), o, 2, 7, 2.0, 1e-2, 0.5, 1, 4.0, 0,
                                                                    1.0, 256, w, wb))
