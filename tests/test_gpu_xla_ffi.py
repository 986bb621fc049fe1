"""GPU parity of the XLA custom-call handlers (include/sbh_xla_ffi.h) with
the C entry points they forward to: call frames built by hand
(tests/xla_ffi_emulator.py stands in for the XLA runtime) for the octree8
build, its softened force and VJP, the stochastic octree8 VJP, the direct
sums, the level-3 build and a Node3 traversal must give byte-identical
outputs to the same operation through sbh_b200 (same kernels, same inputs).
Scratch comes from the emulated XLA allocator (torch memory) or, for a
runtime without one, from cudaMallocAsync; either way nothing stays
allocated after the call."""
import numpy as np
import pytest
import torch

import sbh_b200 as B
import sbh_workloads as W
from xla_ffi_emulator import DT_F32, DT_U8, FakeXla

pytestmark = pytest.mark.gpu


def _torch_alloc():
    def alloc(size):
        t = torch.empty(size, dtype=torch.uint8, device="cuda")
        return t.data_ptr(), t
    return alloc


def _buf(t):
    dt = DT_U8 if t.dtype == torch.uint8 else DT_F32
    return dt, t.data_ptr(), tuple(t.shape)


def _runtime(with_allocator):
    return FakeXla(stream=torch.cuda.current_stream().cuda_stream,
                   allocate=_torch_alloc() if with_allocator else None)


SOFT = dict(beta=np.float32(2.0), softening_scale=np.float32(1e-2), cutoff_scale=np.float32(1.5),
            prune_enabled=np.int32(0), prune_r_cut_mult=np.float32(4.0), periodic=np.int32(0),
            box_length=np.float32(1.0), threads=np.int32(256))


@pytest.mark.parametrize("with_allocator", [True, False])
def test_octree8_build_force_and_vjp_handlers_match_entry_points(cuda, with_allocator):
    L = B.lib()
    x = _runtime(with_allocator)
    p, m = W.plummer(20000, seed=31)
    rng = np.random.default_rng(2)
    nrm = rng.normal(size=p.shape).astype(np.float32)
    P, N, M = (torch.as_tensor(a, device=cuda) for a in (p, nrm, m))
    MN = torch.as_tensor(p.min(0) - np.float32(1e-3), device=cuda)
    MX = torch.as_tensor(p.max(0) + np.float32(1e-3), device=cuda)
    depth = 5
    total = B._octree8_total_nodes(depth)
    leaf = torch.full((p.shape[0] * 32,), 7, dtype=torch.uint8, device=cuda)
    node = torch.full((total * 104,), 7, dtype=torch.uint8, device=cuda)
    con = torch.full((total * 32,), 7, dtype=torch.uint8, device=cuda)
    x.call(L.sbh_build_octree8_buffers_ffi, [_buf(P), _buf(N), _buf(M), _buf(MN), _buf(MX)],
           [_buf(leaf), _buf(node), _buf(con)], dict(max_depth=np.int32(depth)))
    wl, wn, wc = B.build_octree8_buffers_with_contrib(p, nrm, m, MN, MX, max_depth=depth)
    torch.cuda.synchronize()
    assert torch.equal(leaf, wl) and torch.equal(node, wn) and torch.equal(con, wc)
    assert not x.live
    if with_allocator:
        assert x.allocations == 1

    q = P[:5000].contiguous()
    cot = torch.as_tensor(rng.normal(size=(5000, 3)).astype(np.float32), device=cuda)
    out = torch.zeros_like(q)
    x.call(L.sbh_barnes_hut_force_octree8_soft_ffi, [_buf(leaf), _buf(node), _buf(q)], [_buf(out)], SOFT)
    kw = dict(beta=2.0, softening_scale=1e-2, cutoff_scale=1.5, prune_enabled=False)
    want = B.softened_barnes_hut_force_octree8(leaf, node, q, **kw)
    torch.cuda.synchronize()
    assert torch.equal(out, want)
    x.call(L.sbh_barnes_hut_force_octree8_soft_vjp_ffi, [_buf(leaf), _buf(node), _buf(q), _buf(cot)], [_buf(out)],
           SOFT)
    want = B.softened_barnes_hut_force_octree8_vjp(leaf, node, q, cot, **kw)
    torch.cuda.synchronize()
    assert torch.equal(out, want)
    plain = {k: SOFT[k] for k in ("beta", "periodic", "box_length", "threads")}
    x.call(L.sbh_barnes_hut_force_octree8_ffi, [_buf(leaf), _buf(node), _buf(q)], [_buf(out)], plain)
    want = B.barnes_hut_force_octree8(leaf, node, q, beta=2.0)
    torch.cuda.synchronize()
    assert torch.equal(out, want)
    st = dict(SOFT, samples_per_subdomain=np.int32(2), seed=np.int32(11))
    x.call(L.sbh_stochastic_bh_force_octree8_soft_vjp_ffi, [_buf(leaf), _buf(node), _buf(q), _buf(cot)],
           [_buf(out)], st)
    want = B.softened_stochastic_barnes_hut_force_octree8_vjp(leaf, node, q, cot, beta=2.0, samples_per_subdomain=2,
                                                              seed=11, softening_scale=1e-2, cutoff_scale=1.5,
                                                              prune_enabled=False)
    torch.cuda.synchronize()
    assert torch.equal(out, want)
    assert not x.live


def test_direct_and_level3_tree_handlers_match_entry_points(cuda):
    L = B.lib()
    x = _runtime(True)
    p, m = W.plummer(3000, seed=32)
    P, M = torch.as_tensor(p, device=cuda), torch.as_tensor(m, device=cuda)
    q = P[:700].contiguous()
    out = torch.zeros_like(q)
    attrs = dict(softening_scale=np.float32(5e-2), cutoff_scale=np.float32(0.9), periodic=np.int32(0),
                 box_length=np.float32(1.0), threads=np.int32(128))
    x.call(L.sbh_direct_force_soft_ffi, [_buf(P), _buf(M), _buf(q)], [_buf(out)], attrs)
    want = B.softened_direct_force(P, M, q, softening_scale=5e-2, cutoff_scale=0.9, threads=128)
    torch.cuda.synchronize()
    assert torch.equal(out, want)
    pot = torch.zeros(700, device=cuda)
    x.call(L.sbh_bruteforce_gravity_ffi, [_buf(P), _buf(M), _buf(q)], [_buf(pot)],
           dict(periodic=np.int32(0), box_length=np.float32(1.0), threads=np.int32(64)))
    want = B.brute_force_gravity(P, M, q)
    torch.cuda.synchronize()
    assert torch.equal(pot, want)
    # level-3 build and a Node3 softened traversal
    Z = torch.zeros_like(P)
    MN = torch.as_tensor(p.min(0) - np.float32(1e-3), device=cuda)
    MX = torch.as_tensor(p.max(0) + np.float32(1e-3), device=cuda)
    nmax = B.octree_level3_max_nodes()
    leaf = torch.zeros(3000 * 32, dtype=torch.uint8, device=cuda)
    node = torch.zeros(nmax * 4272, dtype=torch.uint8, device=cuda)
    con = torch.zeros(nmax * 32, dtype=torch.uint8, device=cuda)
    x.call(L.sbh_build_octree_level3_buffers_ffi, [_buf(P), _buf(Z), _buf(M), _buf(MN), _buf(MX)],
           [_buf(leaf), _buf(node), _buf(con)], {})
    wl, wn, wc = B.build_octree_buffers_with_contrib(P, Z, M, MN, MX)
    torch.cuda.synchronize()
    assert torch.equal(leaf, wl) and torch.equal(node, wn) and torch.equal(con, wc)
    x.call(L.sbh_barnes_hut_force_soft_ffi_3d, [_buf(leaf), _buf(node), _buf(q)], [_buf(out)],
           dict(beta=np.float32(2.0), softening_scale=np.float32(5e-2), cutoff_scale=np.float32(0.9),
                periodic=np.int32(0), box_length=np.float32(1.0), threads=np.int32(64)))
    want = B.softened_barnes_hut_force(leaf, node, q, beta=2.0, softening_scale=5e-2, cutoff_scale=0.9, threads=64)
    torch.cuda.synchronize()
    assert torch.equal(out, want)
    assert not x.live
