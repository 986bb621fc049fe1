"""Parity and accuracy at the benchmark configurations' own sizes.

* Config 2a's system, N = 2^20 Plummer (a = 1, r < 10a, m = 1/N), through the
  reference-layout octree8 path at depth 7:
  - the build against the reference plugin's build (src/sbh_ffi.cu:1039-1420,
    compiled unmodified into oracle/_ref/libsbh_ref_gpu.so) on the same
    inputs: every topology field and the cell geometry bit-exact, each leaf
    cell holding the same multiset of particle records, monopoles within the
    FP32 reordering tolerance; the number of particles the fast-math
    quantisation puts in another cell than the IEEE oracle is reported;
  - the softened force and its VJP at 4,096 of the particles against the
    reference's kernels (src/sbh_ffi.cu:1995-2042, 2092-2144) on the same
    buffers, within 1e-5 relative L2;
  - the stochastic estimator and its VJP (32 paths per subdomain, fixed
    seed, src/sbh_ffi.cu:2146-2442) at the same queries: every row within
    1e-4 of the reference's.
* Config 1: N = 10,000 uniform in the unit cube, eps = 1e-3, theta = 0.5,
  leaf size 8: the native tree and the octree8 path against the FP64 direct
  sum, the reference's CPU Tree3D<8,1> beside them.
* Config 3: the full gradient of L = sum_i w_i . a_i on the native tree
  (positions and masses, N = 2^20 Plummer, theta = 0.5) against float64
  central finite differences (h = 1e-4, Richardson-extrapolated with h / 2)
  of the same frozen plan on a seeded 4,096-particle subset; the gradient's distance to the exact direct-sum
  gradient; and the query-side term against the FP64 direct query-side VJP,
  beside the reference's octree8 VJP on the same targets.

* Config 4 at its size (256 Plummer systems, N log-uniform in [1e3, 2e5],
  11.6M particles): the forest's force walk in one launch equals each
  system walked on its own; the fused force + adjoint of the forest equals
  the separate systems' for the largest and the smallest system.
* Config 2b's sources: the winding number of 262,144 oriented points on the
  ellipsoid (1, 0.7, 0.5) on the native tree, at 65,536 of the
  configuration's uniform queries: value and full adjoint against the
  oracle's float64 evaluation of the same plan, value against the FP64
  direct sum.

Each test prints the figures it checks (pytest -s shows them).
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

N1M = 1 << 20
EPS = 1e-3
BETA = 2.0


def _t(a, dev, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), device=dev, dtype=dtype)


def _S():
    return torch.cuda.current_stream().cuda_stream


def _node_fields(node):
    a = node.reshape(-1, 104)
    u = a[:, :48].copy().view(np.uint32)
    return dict(u=u, mask=a[:, 48], depth=a[:, 49], is_leaf=a[:, 50], geom=a[:, 52:72].copy().view(np.float32),
                contrib=a[:, 72:104].copy().view(np.float32))


@pytest.fixture(scope="module")
def plummer_1m():
    p, m = W.plummer(N1M, seed=2024)
    rng = np.random.default_rng(77)
    idx = np.sort(rng.choice(N1M, 4096, replace=False))
    w = rng.normal(size=p.shape).astype(np.float32)
    return p, m, w, idx


@needs_ref
def test_octree8_depth7_build_and_traversals_at_2e20_match_reference(cuda, plummer_1m):
    p, m, w, idx = plummer_1m
    depth = 7
    nrm = np.random.default_rng(5).normal(size=p.shape).astype(np.float32)
    mn = (p.min(0) - np.float32(1e-3)).astype(np.float32)
    mx = (p.max(0) + np.float32(1e-3)).astype(np.float32)
    leaf, node, contrib = B.build_octree8_buffers_with_contrib(p, nrm, m, mn, mx, max_depth=depth)
    total = O.octree8_total_nodes(depth)
    L = O.refgpu()
    rleaf = torch.zeros(N1M * 32, dtype=torch.uint8, device=cuda)
    rnode = torch.zeros(total * 104, dtype=torch.uint8, device=cuda)
    rcon = torch.zeros(total * 32, dtype=torch.uint8, device=cuda)
    P, NR, M, MN, MX = (_t(a, cuda) for a in (p, nrm, m, mn, mx))
    O.refgpu_check(L.ref_build_octree8(_S(), P.data_ptr(), NR.data_ptr(), M.data_ptr(), N1M, MN.data_ptr(),
                                       MX.data_ptr(), rleaf.data_ptr(), rleaf.numel(), rnode.data_ptr(), rnode.numel(),
                                       rcon.data_ptr(), rcon.numel(), depth))
    torch.cuda.synchronize()
    a, b = _node_fields(node.cpu().numpy()), _node_fields(rnode.cpu().numpy())
    # start, end, parent, first_child, child[8]; mask, depth, is_leaf; centre, half size, diameter
    np.testing.assert_array_equal(a["u"], b["u"])
    for k in ("mask", "depth", "is_leaf", "geom"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    np.testing.assert_allclose(a["contrib"], b["contrib"], rtol=2e-5, atol=1e-6)
    # leaf cells (depth 7) hold the same records: sort each cell's records
    start, end = a["u"][:, 0].astype(np.int64), a["u"][:, 1].astype(np.int64)
    cells = np.nonzero(a["depth"] == depth)[0]
    seg = np.repeat(np.arange(cells.size), end[cells] - start[cells])
    assert seg.size == N1M
    la = leaf.cpu().numpy().reshape(-1, 8 * 4).view(np.float32)
    lb = rleaf.cpu().numpy().reshape(-1, 8 * 4).view(np.float32)

    def canon(rec):
        order = np.lexsort(tuple(rec[:, c] for c in range(7, -1, -1)) + (seg,))
        return rec[order]

    np.testing.assert_array_equal(canon(la), canon(lb))
    # fast-math quantisation (the reference's --use_fast_math) against IEEE
    # division in the oracle: particles counted in a different depth-7 cell
    _, onode, _, _, _ = O.build_octree8(p, nrm, m, mn, mx, depth)
    o = _node_fields(onode)
    ours_count = (end - start)[cells]
    oracle_count = (o["u"][:, 1].astype(np.int64) - o["u"][:, 0].astype(np.int64))[cells]
    moved = int(np.abs(ours_count - oracle_count).sum() // 2)
    print(f"\n[octree8 2^20 depth 7] topology and geometry bit-exact vs the reference build; "
          f"{cells.size} leaf cells with equal multisets; {moved} of {N1M} particles in another cell than the "
          f"IEEE oracle")
    assert moved <= 1e-3 * N1M

    # softened force and its VJP at 4,096 particles, against the reference kernels on the same buffers
    q, cot = p[idx], w[idx]
    Q, C = _t(q, cuda), _t(cot, cuda)
    nq = q.shape[0]
    span = float((p.max(0) - p.min(0)).max())
    cut = 1e6 * span  # the reference's "no cutoff" convention: 1e6 box lengths
    lp, lb_, np_, nb = leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel()
    rf = torch.zeros((nq, 3), device=cuda)
    O.refgpu_check(L.ref_bh_force_octree8_soft(_S(), lp, lb_, np_, nb, Q.data_ptr(), nq, rf.data_ptr(), BETA, EPS, cut,
                                               0, 4.0, 0, 1.0, 256))
    rv = torch.zeros((nq, 3), device=cuda)
    O.refgpu_check(L.ref_bh_force_octree8_soft_vjp(_S(), lp, lb_, np_, nb, Q.data_ptr(), nq, C.data_ptr(),
                                                   rv.data_ptr(), BETA, EPS, cut, 0, 4.0, 0, 1.0, 256))
    kw = dict(beta=BETA, softening_scale=EPS, cutoff_scale=cut, prune_enabled=False, check_status=True)
    f = B.softened_barnes_hut_force_octree8(leaf, node, q, **kw)
    v = B.softened_barnes_hut_force_octree8_vjp(leaf, node, q, cot, **kw)
    torch.cuda.synchronize()
    ef = rel_l2(f.cpu().numpy(), rf.cpu().numpy())
    ev = rel_l2(v.cpu().numpy(), rv.cpu().numpy())
    print(f"[octree8 2^20 depth 7, 4096 queries] force vs reference kernel {ef:.2e}, VJP {ev:.2e}")
    assert ef < 1e-5
    assert ev < 1e-5

    # the stochastic estimator (MLPCV, 32 paths per subdomain: config 2a's "32 samples") and its VJP at
    # the same queries, same seed: the same curand streams, so every row on the reference's paths
    sf = torch.zeros((nq, 3), device=cuda)
    O.refgpu_check(L.ref_stochastic_bh_force_octree8(_S(), 1, lp, lb_, np_, nb, Q.data_ptr(), nq, sf.data_ptr(), 32, 7,
                                                     BETA, EPS, cut, 0, 4.0, 0, 1.0, 256))
    sv = torch.zeros((nq, 3), device=cuda)
    O.refgpu_check(L.ref_stochastic_bh_force_octree8_vjp(_S(), 1, lp, lb_, np_, nb, Q.data_ptr(), nq, C.data_ptr(),
                                                         sv.data_ptr(), 32, 7, BETA, EPS, cut, 0, 4.0, 0, 1.0, 256))
    skw = dict(samples_per_subdomain=32, seed=7, beta=BETA, softening_scale=EPS, cutoff_scale=cut,
               prune_enabled=False, check_status=True)
    gf = B.softened_stochastic_barnes_hut_force_octree8(leaf, node, q, **skw)
    gv = B.softened_stochastic_barnes_hut_force_octree8_vjp(leaf, node, q, cot, **skw)
    torch.cuda.synchronize()
    for tag, got, want in (("force", gf, sf), ("VJP", gv, sv)):
        g_, w_ = got.cpu().numpy(), want.cpu().numpy()
        # rows relative to their own norm, floored at 1% of the rows' RMS norm (a row that nearly
        # cancels would otherwise inflate its FP32 rounding; a different path is an O(1) error)
        nrm_ = np.linalg.norm(w_.astype(np.float64), axis=1)
        row = np.linalg.norm(g_ - w_, axis=1) / np.maximum(nrm_, 1e-2 * np.sqrt(np.mean(nrm_ ** 2)))
        print(f"[stochastic octree8 2^20 depth 7, 4096 queries, 32 paths] {tag}: worst row {row.max():.2e}, "
              f"rel-L2 {rel_l2(g_, w_):.2e}")
        assert row.max() < 1e-4


def test_config1_uniform_10k_accuracy_vs_fp64_direct(cuda):
    p, m = W.uniform_cube(10000, seed=1)
    want = O.direct_force_soft(p, m, p, EPS)
    native = B.NativeTree().build(p, m, leaf_size=8, with_adjoint=False).force(beta=BETA, softening=EPS)
    e_native = rel_l2(native.cpu().numpy(), want)
    e_mono = rel_l2(B.NativeTree().build(p, m, leaf_size=8, with_adjoint=False)
                    .force(beta=BETA, softening=EPS, quadrupole=False).cpu().numpy(), want)
    span = float((p.max(0) - p.min(0)).max())
    e_o8 = {}
    for depth in (3, 4):
        leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, max_depth=depth)
        f = B.softened_barnes_hut_force_octree8(leaf, node, p, beta=BETA, softening_scale=EPS, cutoff_scale=1e6 * span,
                                                prune_enabled=False, check_status=True)
        e_o8[depth] = rel_l2(f.cpu().numpy(), want)
    line = (f"\n[config 1] rel-L2 vs FP64 direct: native leaf 8 {e_native:.2e} (monopole only {e_mono:.2e}); "
            f"octree8 depth 3 {e_o8[3]:.2e}, depth 4 {e_o8[4]:.2e}")
    if O.available("libsbh_ref_cpu.so"):
        ref, _ = O.RefTree3D(p, m, variant=0).eval(p, BETA, O.REF_K_SOFT_FORCE, eps=EPS)
        e_ref = rel_l2(ref, want)
        line += f"; reference CPU Tree3D<8,1> {e_ref:.2e}"
        assert e_native < e_ref
    print(line)
    assert e_native < 1e-4
    assert e_mono < 1e-3
    assert max(e_o8.values()) < 1e-3


@needs_ref
def test_config3_gradient_vs_fp64_finite_differences_at_2e20(cuda, plummer_1m):
    p, m, w, idx = plummer_1m
    G = B.native_group_size()
    t = B.NativeTree().build(p, m, leaf_size=16, with_adjoint=True)
    _, gx, gm = t.force_vjp(w, beta=BETA, softening=EPS, want_force=False)
    gq = t.query_side_gradient()
    torch.cuda.synchronize()
    gx, gm, gq = gx.cpu().numpy()[idx], gm.cpu().numpy()[idx], gq.cpu().numpy()[idx]
    st = t.stats()
    T = O.NativeTree(p, m, leaf_size=16)
    with O.native_quadrupole_radius(B.QUADRUPOLE_RADIUS), O.native_quadrupole_linear(B.QUADRUPOLE_LINEAR):
        count = T.plan(BETA, G)
    assert count == st["far"] + st["near"], "the GPU walk and the oracle took different plans"
    # h = 1e-4 central differences carry an O(h^2) truncation error of about
    # 1e-3 here (softened pairs closer than 1e-2); Richardson extrapolation
    # with h / 2, (4 D(h/2) - D(h)) / 3, removes it (it then agrees with
    # h = 1e-6 to 1e-7 on the oracle alone)
    fx, fm = T.finite_differences(w, EPS, idx, hx=1e-4, hm_rel=1e-4, quad=True)
    fx2, fm2 = T.finite_differences(w, EPS, idx, hx=5e-5, hm_rel=5e-5, quad=True)
    rx, rm = (4.0 * fx2 - fx) / 3.0, (4.0 * fm2 - fm) / 3.0
    e_x, e_m = rel_l2(gx, rx), rel_l2(gm, rm)
    e_x1, e_m1 = rel_l2(gx, fx), rel_l2(gm, fm)
    ex, em = O.direct_full_adjoint(p, m, w, EPS, idx=idx)
    a_x, a_m = rel_l2(gx, ex), rel_l2(gm, em)
    # query-side term: native and the reference's octree8 VJP (depth 7) against the FP64 direct query-side VJP.
    # With the query at a source's position the direct VJP holds the self pair's term -m J(0)^T w =
    # -m (eps^2 + 1e-12)^(-3/2) w (the query moves, the source stays); in self-gravity the pair's
    # query and source sides cancel, so the native walk leaves it out: it is added back for the comparison.
    want_q = O.direct_force_soft_vjp(p, m, p[idx], w[idx], EPS)
    self_q = -(m[idx].astype(np.float64) * (EPS * EPS + 1e-12) ** -1.5)[:, None] * w[idx].astype(np.float64)
    e_q = rel_l2(gq, want_q - self_q)
    leaf, node = B.build_octree8_buffers(p, np.zeros_like(p), m, max_depth=7)
    Q, C = _t(p[idx], cuda), _t(w[idx], cuda)
    rv = torch.zeros((idx.size, 3), device=cuda)
    span = float((p.max(0) - p.min(0)).max())
    O.refgpu_check(O.refgpu().ref_bh_force_octree8_soft_vjp(_S(), leaf.data_ptr(), leaf.numel(), node.data_ptr(),
                                                            node.numel(), Q.data_ptr(), idx.size, C.data_ptr(),
                                                            rv.data_ptr(), BETA, EPS, 1e6 * span, 0, 4.0, 0, 1.0, 256))
    torch.cuda.synchronize()
    e_ref = rel_l2(rv.cpu().numpy(), want_q)
    print(f"\n[config 3, 2^20 Plummer, 4096 particles] native gradient vs FP64 central FD of the frozen plan "
          f"(h = 1e-4, Richardson with h/2): positions {e_x:.2e}, masses {e_m:.2e} (plain h = 1e-4: {e_x1:.2e}, "
          f"{e_m1:.2e}); vs the exact direct-sum gradient: positions {a_x:.2e}, masses {a_m:.2e}; query-side "
          f"term vs FP64 direct query-side VJP: native {e_q:.2e}, reference octree8 VJP (depth 7) {e_ref:.2e}")
    assert e_x < 1e-4
    assert e_m < 1e-4
    assert e_x1 < 1e-2
    assert a_x < 1e-3 and a_m < 3e-3
    assert e_q < 1e-4


def test_config2b_winding_number_parity_at_size(cuda):
    pts, nrm, wgt = W.ellipsoid_surface(262144, seed=2)
    q = W.uniform_box_queries(1048576, seed=3)
    q = np.ascontiguousarray(q[np.random.default_rng(4).choice(q.shape[0], 65536, replace=False)])
    u = np.random.default_rng(5).normal(size=q.shape[0]).astype(np.float32)
    t = B.NativeTree().build(pts, wgt, normals=nrm, leaf_size=16, with_adjoint=True)
    w, gq, gp, gn, gm = t.winding_number_vjp(q, u, beta=2.0, want_value=True)
    T = O.NativeTree(pts, wgt, leaf_size=16)
    T.wn_plan(q, 2.0)
    want_w = T.wn_eval(nrm)
    dq, dp, dn, dm = T.wn_adjoint(nrm, u)
    errs = dict(value=rel_l2(w.cpu().numpy(), want_w), dq=rel_l2(gq.cpu().numpy(), dq),
                dp=rel_l2(gp.cpu().numpy(), dp), dn=rel_l2(gn.cpu().numpy(), dn), dm=rel_l2(gm.cpu().numpy(), dm))
    sub = np.arange(0, q.shape[0], 64)
    direct = O.direct_winding_number(pts, nrm, wgt, q[sub])
    errs["vs_fp64_direct"] = rel_l2(w.cpu().numpy()[sub], direct)
    print("config 2b parity at 262,144 sources / 65,536 queries:", errs)
    assert errs["value"] < 1e-5
    for k in ("dq", "dp", "dn", "dm"):
        assert errs[k] < 1e-4
    assert errs["vs_fp64_direct"] < 5e-3


def test_config4_forest_equals_separate_systems_at_size(cuda):
    systems, sizes = W.forest(256, 1000, 200000, seed=0)
    pts = torch.tensor(np.concatenate([s_[0] for s_ in systems]), device=cuda)
    ms = torch.tensor(np.concatenate([s_[1] for s_ in systems]), device=cuda)
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    w = torch.randn(pts.shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(6))
    forest = B.NativeTree().build(pts, ms, system_offsets=offs, leaf_size=16)
    f_all = forest.force(beta=BETA, softening=EPS)
    _, gx_all, gm_all = forest.force_vjp(w, beta=BETA, softening=EPS, want_force=False)
    tree = B.NativeTree()
    worst = 0.0
    for i in range(len(systems)):
        a, b = int(offs[i]), int(offs[i + 1])
        tree.build(pts[a:b], ms[a:b], leaf_size=16)
        fi = tree.force(beta=BETA, softening=EPS)
        # same tree and groups; node moments differ in the last bits because the forest's FP64
        # prefix sums also carry the earlier systems
        worst = max(worst, rel_l2(f_all[a:b].cpu().numpy(), fi.cpu().numpy()))
    checked = []
    for i in (int(np.argmax(sizes)), int(np.argmin(sizes))):
        a, b = int(offs[i]), int(offs[i + 1])
        tree.build(pts[a:b], ms[a:b], leaf_size=16)
        _, gxi, gmi = tree.force_vjp(w[a:b], beta=BETA, softening=EPS, want_force=False)
        checked.append((rel_l2(gx_all[a:b].cpu().numpy(), gxi.cpu().numpy()),
                        rel_l2(gm_all[a:b].cpu().numpy(), gmi.cpu().numpy())))
    print(f"config 4 forest ({int(offs[-1])} particles, 256 systems): worst system force {worst:.2e}; "
          f"adjoint (positions, masses) largest {checked[0][0]:.2e} {checked[0][1]:.2e}, "
          f"smallest {checked[1][0]:.2e} {checked[1][1]:.2e}")
    assert worst < 1e-6
    for gx_err, gm_err in checked:
        assert gx_err < 1e-5 and gm_err < 1e-5
