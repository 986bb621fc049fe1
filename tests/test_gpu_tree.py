"""GPU parity of the level-3 builder and the Node2 / Node3 targets
(src/sbh_ffi.cu:192-397, 1422-1680, 2444-3131) against the reference's own
kernels on the same buffers. The deeper Node3 / Node2 trees come from the
reference's CPU builders (Tree3D<1,3>, Tree2D<1,3> compiled into oracle/_ref),
as the reference's own Python does (python/jax_sbh_ffi.py:658-742)."""
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


def _u8(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), device=dev, dtype=torch.uint8)


def node3_fields(nb):
    a = np.asarray(nb.cpu() if isinstance(nb, torch.Tensor) else nb).reshape(-1, 4272)
    u64 = a[:, :32].copy().view(np.uint64)
    f = a[:, 32:92].copy().view(np.float32)
    mask = a[:, 96:160].copy().view(np.uint64)
    child = a[:, 160:4256].copy().view(np.uint64)
    ints = a[:, 4256:4268].copy().view(np.int32)
    return dict(u64=u64, f=f, mask=mask, child=child, ints=ints, leaf=a[:, 4268])


def ref_level3(dev, p, nrm, m, mn, mx):
    L = O.refgpu()
    n = p.shape[0]
    leaf = torch.zeros(n * 32, dtype=torch.uint8, device=dev)
    node = torch.zeros(513 * 4272, dtype=torch.uint8, device=dev)
    contrib = torch.zeros(513 * 32, dtype=torch.uint8, device=dev)
    P, N, M, MN, MX = _t(p, dev), _t(nrm, dev), _t(m, dev), _t(mn, dev), _t(mx, dev)
    O.refgpu_check(L.ref_build_octree_level3(_S(), P.data_ptr(), N.data_ptr(), M.data_ptr(), n, MN.data_ptr(),
                                             MX.data_ptr(), leaf.data_ptr(), leaf.numel(), node.data_ptr(),
                                             node.numel(), contrib.data_ptr(), contrib.numel()))
    torch.cuda.synchronize()
    return leaf, node, contrib


@needs_ref
def test_level3_build_matches_reference(cuda):
    p, m = W.plummer(6000, seed=3)
    nrm = np.random.default_rng(1).normal(size=p.shape).astype(np.float32)
    mn = p.min(0) - np.float32(1e-3)
    mx = p.max(0) + np.float32(1e-3)
    leaf, node, contrib = B.build_octree_buffers_with_contrib(p, nrm, m, mn, mx)
    rleaf, rnode, rcontrib = ref_level3(cuda, p, nrm, m, mn, mx)
    a, b = node3_fields(node), node3_fields(rnode)
    np.testing.assert_array_equal(a["u64"], b["u64"])
    np.testing.assert_array_equal(a["mask"], b["mask"])
    np.testing.assert_array_equal(a["child"], b["child"])
    np.testing.assert_array_equal(a["ints"], b["ints"])
    np.testing.assert_array_equal(a["leaf"], b["leaf"])
    np.testing.assert_array_equal(a["f"][:, :7], b["f"][:, :7])  # bounds and diameter
    # contrib: the reference sums with FP32 atomics (its root mass here is
    # 0.99995 instead of 1); ours sums in FP64
    np.testing.assert_allclose(a["f"][:, 7:], b["f"][:, 7:], rtol=2e-4, atol=2e-6)
    assert abs(float(a["f"][0, 13]) - float(m.astype(np.float64).sum())) < 1e-6
    la = leaf.cpu().numpy().reshape(-1, 32).copy().view(np.float32)
    lb = rleaf.cpu().numpy().reshape(-1, 32).copy().view(np.float32)
    for s, e in b["u64"][1:, :2]:
        if e > s:
            assert sorted(map(tuple, la[s:e])) == sorted(map(tuple, lb[s:e]))


def _ref_tree_call(fn_name, dev, dim, leaf, node, q, *args, vec):
    L = O.refgpu()
    nq = q.shape[0]
    out = torch.zeros((nq, dim) if vec else nq, device=dev)
    Q = _t(q, dev)
    O.refgpu_check(getattr(L, fn_name)(_S(), dim, leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                       Q.data_ptr(), nq, out.data_ptr(), *args))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@needs_ref
@pytest.mark.parametrize("threads", [64, 256, 96])
def test_node3_level3_traversals_match_reference(cuda, threads):
    p, m = W.plummer(3000, seed=5)
    p = p * np.float32(0.3)
    leaf, node, contrib = B.build_octree_buffers_with_contrib(p, np.zeros_like(p), m)
    rng = np.random.default_rng(2)
    q = np.concatenate([p[:400], rng.uniform(-8, 8, (200, 3)).astype(np.float32)])
    for beta in (2.0, 0.3):
        want = _ref_tree_call("ref_barnes_hut_gravity", cuda, 3, leaf, node, q, beta, 0, 1.0, threads, vec=False)
        got = B.barnes_hut_gravity(leaf, node, q, beta=beta, threads=threads).cpu().numpy()
        assert rel_l2(got, want) < 1e-6
        want = _ref_tree_call("ref_barnes_hut_force", cuda, 3, leaf, node, q, beta, 0, 1.0, threads, vec=True)
        got = B.barnes_hut_force(leaf, node, q, beta=beta, threads=threads).cpu().numpy()
        assert rel_l2(got, want) < 1e-6
        want = _ref_tree_call("ref_barnes_hut_force_soft", cuda, 3, leaf, node, q, beta, 5e-2, 1.5, 0, 1.0, threads,
                              vec=True)
        got = B.softened_barnes_hut_force(leaf, node, q, beta=beta, softening_scale=5e-2, cutoff_scale=1.5,
                                          threads=threads).cpu().numpy()
        assert rel_l2(got, want) < 1e-6


@needs_ref
def test_node3_and_node2_cpu_built_trees_match_reference(cuda):
    p, m = W.uniform_cube(1500, seed=7)
    t3 = O.RefTree3D(p, m, variant=2)
    leaf3, node3 = _u8(t3.leaf_bytes(), cuda), _u8(t3.node_bytes(), cuda)
    q = p[:300]
    want = _ref_tree_call("ref_barnes_hut_force", cuda, 3, leaf3, node3, q, 2.0, 0, 1.0, 64, vec=True)
    got = B.barnes_hut_force(leaf3, node3, q, beta=2.0, threads=64).cpu().numpy()
    assert rel_l2(got, want) < 1e-6
    p2 = p[:, :2].copy()
    t2 = O.RefTree2D(p2, m)
    leaf2, node2 = _u8(t2.leaf_bytes(), cuda), _u8(t2.node_bytes(), cuda)
    q2 = p2[:300]
    want = _ref_tree_call("ref_barnes_hut_gravity", cuda, 2, leaf2, node2, q2, 2.0, 0, 1.0, 64, vec=False)
    got = B.barnes_hut_gravity(leaf2, node2, q2, beta=2.0, threads=64).cpu().numpy()
    assert rel_l2(got, want) < 1e-6
    want = _ref_tree_call("ref_barnes_hut_force_soft", cuda, 2, leaf2, node2, q2, 2.0, 5e-2, 1.5, 0, 1.0, 64, vec=True)
    got = B.softened_barnes_hut_force(leaf2, node2, q2, beta=2.0, softening_scale=5e-2, cutoff_scale=1.5,
                                      threads=64).cpu().numpy()
    assert rel_l2(got, want) < 1e-6


@needs_ref
@pytest.mark.parametrize("dim", [2, 3])
def test_tree_mlpcv_fixed_seed_matches_reference(cuda, dim):
    p, m = W.uniform_cube(1200, seed=9)
    if dim == 3:
        t = O.RefTree3D(p, m, variant=2)
    else:
        p = p[:, :2].copy()
        t = O.RefTree2D(p, m)
    leaf, node, contrib = _u8(t.leaf_bytes(), cuda), _u8(t.node_bytes(), cuda), _u8(t.contrib_bytes(), cuda)
    q = p[:256]
    L = O.refgpu()
    Q = _t(q, cuda)
    for kernel, fn, vec in ((B.TREE_POTENTIAL, "ref_stochastic_bh_gravity", False),
                            (B.TREE_FORCE, "ref_stochastic_bh_force", True)):
        out = torch.zeros((256, dim) if vec else 256, device=cuda)
        O.refgpu_check(getattr(L, fn)(_S(), dim, leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                      contrib.data_ptr(), contrib.numel(), Q.data_ptr(), 256, out.data_ptr(), 2, 5, 0,
                                      1.0, 64))
        torch.cuda.synchronize()
        got = B._stochastic_tree_call(kernel, leaf, node, contrib, q, 2, 5, 0.0, 1.0, False, 1.0, 64).cpu().numpy()
        want = out.cpu().numpy()
        row = np.abs(got - want).reshape(256, -1).max(1) / np.maximum(np.abs(want).reshape(256, -1).max(1), 1e-30)
        # same curand streams: every row on the reference's sampled paths
        assert row.max() < 1e-4, f"{int((row >= 1e-4).sum())} rows differ, worst {row.max():.2e}"


def test_node3_winding_number_and_direct_limit(cuda):
    pts, nrm, w = W.ellipsoid_surface(3000, seed=4)
    t = O.RefTree3D(pts, w, normals=nrm, variant=2)
    leaf, node = _u8(t.leaf_bytes(), cuda), _u8(t.node_bytes(), cuda)
    q = W.uniform_box_queries(512, seed=8)
    got = B.barnes_hut_winding_number(leaf, node, q, beta=1e30).cpu().numpy()
    want = O.direct_winding_number(pts, nrm, w, q)
    assert rel_l2(got, want) < 1e-5
    bh = B.barnes_hut_winding_number(leaf, node, q, beta=2.0).cpu().numpy()
    assert np.abs(bh - want).max() < 5e-2


@pytest.mark.parametrize("dist", ["uniform", "plummer", "clustered", "one", "dupes"])
def test_quadtree_build_matches_reference_cpu_builder(cuda, dist):
    """The GPU quadtree builder gives the bytes of the reference's CPU builder
    Tree2D<1,3> (sbh.Quadtree3) for leaves, nodes and contrib records."""
    rng = np.random.default_rng(61)
    if dist == "uniform":
        p, m = W.uniform_cube(4000, seed=51)
    elif dist == "plummer":
        p, m = W.plummer(20000, seed=52)
    elif dist == "clustered":
        p, m = W.plummer(3000, seed=53)
        p = p * np.float32(1e-3)  # deep chains of single-child nodes
    elif dist == "one":
        p, m = W.uniform_cube(1, seed=54)
    else:
        p, m = W.uniform_cube(500, seed=55)
        p = np.concatenate([p, np.repeat(p[:2], 3, axis=0)])  # identical records: depth-100 leaves
        m = np.full(p.shape[0], 1.0 / p.shape[0], np.float32)
    p = np.ascontiguousarray(p[:, :2])
    nrm = rng.normal(size=p.shape).astype(np.float32)
    if dist == "dupes":
        nrm[500:] = nrm[np.array([0, 0, 0, 1, 1, 1])]
    mn = (p.min(0) - np.float32(1e-3)).astype(np.float32)
    mx = (p.max(0) + np.float32(1e-3)).astype(np.float32)
    t = O.RefTree2D(p, m, normals=nrm, min_corner=mn, max_corner=mx, alpha=0.75)
    leaf, node, contrib = B.build_quadtree_buffers_with_contrib(p, nrm, m, mn, mx, alpha=0.75)
    assert node.numel() == t.num_nodes * B.NODE2_BYTES
    np.testing.assert_array_equal(leaf.cpu().numpy(), t.leaf_bytes())
    # every byte but the struct padding (76-79 after the contrib record and
    # 613-615 after is_leaf), which the reference's node copies leave
    # unspecified and which we write as zeros
    keep = np.ones(B.NODE2_BYTES, bool)
    keep[76:80] = False
    keep[613:616] = False
    a = node.cpu().numpy().reshape(-1, B.NODE2_BYTES)[:, keep]
    b = t.node_bytes().reshape(-1, B.NODE2_BYTES)[:, keep]
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(contrib.cpu().numpy(), t.contrib_bytes())


def test_quadtree_buffers_drive_the_2d_targets(cuda):
    p, m = W.plummer(6000, seed=57)
    p = np.ascontiguousarray(p[:, :2])
    leaf, node, contrib = B.build_quadtree_buffers_with_contrib(p, np.zeros_like(p), m)
    q = p[:256]
    got = B.barnes_hut_force(leaf, node, q, beta=1e30, threads=64).cpu().numpy()
    r = q[:, None, :].astype(np.float64) - p[None, :, :].astype(np.float64)
    d = np.sqrt((r * r).sum(-1))
    want = (-m[None, :, None] * r / (d[..., None] + 0.1) ** 3).sum(1)
    assert rel_l2(got, want) < 1e-5
    bh = B.barnes_hut_force(leaf, node, q, beta=2.0, threads=64).cpu().numpy()
    assert rel_l2(bh, want) < 2e-2
    s = B.stochastic_barnes_hut_force(leaf, node, contrib, q, samples_per_subdomain=2, seed=1, threads=64)
    assert torch.isfinite(s).all()


@pytest.mark.parametrize("dist", ["uniform", "plummer", "clustered", "one"])
def test_adaptive_octree_build_matches_reference_cpu_builder(cuda, dist):
    """build_octree_buffers(backend="cpu"): the GPU builder of the adaptive
    Tree3D<1,3> gives the bytes of the reference's CPU builder sbh.Octree3."""
    rng = np.random.default_rng(62)
    if dist == "uniform":
        p, m = W.uniform_cube(3000, seed=71)
    elif dist == "plummer":
        p, m = W.plummer(6000, seed=72)
    elif dist == "clustered":
        p, m = W.plummer(1500, seed=73)
        p = p * np.float32(1e-3)
    else:
        p, m = W.uniform_cube(1, seed=74)
    nrm = rng.normal(size=p.shape).astype(np.float32)
    mn = (p.min(0) - np.float32(1e-3)).astype(np.float32)
    mx = (p.max(0) + np.float32(1e-3)).astype(np.float32)
    t = O.RefTree3D(p, m, normals=nrm, min_corner=mn, max_corner=mx, variant=2, alpha=1.0)
    leaf, node, contrib = B.build_octree_buffers_with_contrib(p, nrm, m, mn, mx, backend="cpu")
    size = B.node3_size()
    assert node.numel() == t.num_nodes * size
    np.testing.assert_array_equal(leaf.cpu().numpy(), t.leaf_bytes())
    keep = np.ones(size, bool)
    keep[92:96] = False  # padding after the contrib record
    keep[4269:4272] = False  # padding after is_leaf
    a = node.cpu().numpy().reshape(-1, size)[:, keep]
    b = t.node_bytes().reshape(-1, size)[:, keep]
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(contrib.cpu().numpy(), t.contrib_bytes())


@pytest.mark.parametrize("dim", [2, 3])
def test_sbh_gpu_module_evaluations_match_reference(cuda, dim):
    """The pybind module sbh_gpu's scalar evaluations (brute force, warp-vote
    BH and MLPCV with seed 0 for every query; gravity potential, winding
    number, smooth distance) against the reference's own templates on the
    same Node2/Node3 buffers."""
    if not HAVE_REF:
        pytest.skip("reference GPU build missing (make -C oracle ref)")
    rng = np.random.default_rng(81)
    p, m = W.uniform_cube(2000, seed=82)
    p = np.ascontiguousarray(p[:, :dim])
    nrm = rng.normal(size=p.shape).astype(np.float32)
    alpha = 3.0
    if dim == 2:
        leaf, node, contrib = B.build_quadtree_buffers_with_contrib(p, nrm, m, alpha=alpha)
    else:
        t = O.RefTree3D(p, m, normals=nrm, variant=2, alpha=alpha)
        leaf, node, contrib = _u8(t.leaf_bytes(), cuda), _u8(t.node_bytes(), cuda), _u8(t.contrib_bytes(), cuda)
    q = rng.uniform(-0.2, 1.2, (300, dim)).astype(np.float32)
    Q = _t(q, cuda)
    L = O.refgpu()
    n = p.shape[0]
    for kind, name in ((0, "gravity"), (3, "wn"), (6, "smoothdist")):
        out = torch.zeros(300, device=cuda)
        O.refgpu_check(L.ref_sbhgpu_brute(_S(), dim, kind, leaf.data_ptr(), n, _t(q.T.copy(), cuda).data_ptr(), 300,
                                          out.data_ptr()))
        torch.cuda.synchronize()
        got, ms = getattr(B, f"eval_brute_force_{name}")(leaf, q)
        assert ms >= 0
        np.testing.assert_allclose(got.cpu().numpy(), out.cpu().numpy(), rtol=1e-6, atol=1e-7)
        for beta in (2.0, 0.5):
            out = torch.zeros(300, device=cuda)
            O.refgpu_check(L.ref_sbhgpu_barnes_hut(_S(), dim, kind, leaf.data_ptr(), node.data_ptr(), Q.data_ptr(),
                                                   300, beta, out.data_ptr()))
            torch.cuda.synchronize()
            got, _ = getattr(B, f"eval_barnes_hut_{name}")(leaf, node, q, beta)
            assert rel_l2(got.cpu().numpy(), out.cpu().numpy()) < 1e-6
        out = torch.zeros(300, device=cuda)
        O.refgpu_check(L.ref_sbhgpu_mlpcv(_S(), dim, kind, leaf.data_ptr(), n, node.data_ptr(), contrib.data_ptr(),
                                          Q.data_ptr(), 300, 2, out.data_ptr()))
        torch.cuda.synchronize()
        got, _ = getattr(B, f"multi_level_prefix_control_variate_{name}")(leaf, node, contrib, q, 2)
        want = out.cpu().numpy()
        # same curand streams: every row on the reference's sampled paths; the
        # error is relative, with values near zero (a winding number far
        # outside) measured against 1% of the outputs' RMS
        rms = float(np.sqrt(np.mean(want.astype(np.float64) ** 2)))
        row = np.abs(got.cpu().numpy() - want) / np.maximum(np.abs(want), 1e-2 * rms)
        assert row.max() < 1e-4, f"{int((row >= 1e-4).sum())} rows differ, worst {row.max():.2e}"
