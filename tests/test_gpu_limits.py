"""Device-side limits of the octree8 traversals on caller-supplied buffers.

The octree8 node buffer crosses the C ABI from the caller, so the traversals
must stay in bounds and terminate on malformed trees (the reference's kernels
would read past their arrays or loop, src/sbh_ffi.cu:1995-2042,2146-2291).
Each test hands a tiny, hand-made node buffer to the kernels and checks the
status bit the kernel records in the workspace:

* a cycle in the child indices: every query pops at most num_nodes nodes and
  the stochastic descent at most 64 levels, then SBH_DEV_ITER_LIMIT;
* a child index past the end of the buffer: skipped, SBH_DEV_BAD_BOUNDS;
* a chain whose nodes list the next node eight times (no cycle, but the DFS
  stack fills): SBH_DEV_STACK_OVERFLOW.

The deterministic traversals run each case twice: 5 queries one thread per
query, and 4,096 queries with the ordered workspace, which a warp walks 32 at
a time down one shared-memory stack (the same caps per warp).

Every index in these buffers is in range or checked by the kernel before use,
and every loop is bounded, so no access leaves the buffers.
"""
import numpy as np
import pytest
import torch

import sbh_b200 as B

pytestmark = pytest.mark.gpu

NODE = 104


def make_nodes(specs):
    """specs: list of dicts with keys child (list of 8 or fewer indices; the
    mask has a bit per listed slot), depth, is_leaf, start, end. Every node
    has its centre at the origin, diameter 1 and contrib mass 1."""
    buf = np.zeros((len(specs), NODE), np.uint8)
    for i, sp in enumerate(specs):
        u = np.zeros(12, np.uint32)
        u[0], u[1], u[2] = sp.get("start", 0), sp.get("end", 0), 0
        kids = sp.get("child", [])
        u[3] = kids[0] if kids else 0xFFFFFFFF
        mask = 0
        for c, k in enumerate(kids):
            u[4 + c] = k
            mask |= 1 << c
        buf[i, :48] = u.view(np.uint8)
        buf[i, 48] = mask
        buf[i, 49] = sp.get("depth", 0)
        buf[i, 50] = sp.get("is_leaf", 0)
        buf[i, 52:72] = np.array([0, 0, 0, 0.5, 1.0], np.float32).view(np.uint8)
        buf[i, 72:104] = np.array([0.01, 0.02, 0.03, 0, 0, 0, 1.0, 1.0], np.float32).view(np.uint8)
    return buf.reshape(-1)


def leaves(n):
    rec = np.zeros((n, 8), np.float32)
    rec[:, 0:3] = np.linspace(-0.3, 0.3, 3 * n, dtype=np.float32).reshape(n, 3)
    rec[:, 6] = 1.0
    return rec.view(np.uint8).reshape(-1)


def run(node_buf, leaf_buf, stochastic=False, nq=5):
    """Traverses nq queries near the origin; nq >= 4096 takes the ordered
    workspace (queries in Morton order, the warp-cooperative kernel)."""
    dev = torch.device("cuda", 0)
    node = torch.as_tensor(node_buf, device=dev)
    leaf = torch.as_tensor(leaf_buf, device=dev)
    q = torch.zeros((nq, 3), dtype=torch.float32, device=dev)
    q[:, 0] = torch.linspace(-0.01, 0.01, nq, device=dev)
    out = torch.full((nq, 3), float("nan"), dtype=torch.float32, device=dev)
    L = B.lib()
    nb = L.sbh_traversal_ordered_workspace_bytes(nq) if nq >= 4096 else L.sbh_traversal_workspace_bytes()
    ws = torch.zeros(int(nb), dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    if stochastic:
        rc = L.sbh_stochastic_bh_force_octree8(s, 0, leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                               q.data_ptr(), nq, out.data_ptr(), 2, 3, 2.0, 0.0, 1.0, 0, 4.0, 0,
                                               1.0, 64, ws.data_ptr(), ws.numel())
    else:
        rc = L.sbh_barnes_hut_force_octree8(s, leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                            q.data_ptr(), nq, out.data_ptr(), 2.0, 0, 1.0, 64, ws.data_ptr(),
                                            ws.numel())
    assert rc == B.SBH_OK, B.last_error()
    torch.cuda.synchronize()
    status = B.read_device_status(ws)
    return status, out.cpu().numpy()


@pytest.mark.parametrize("nq", [5, 4096])
def test_cycle_in_child_indices_stops_with_iter_limit(cuda, nq):
    # 0 -> 1 -> 0: the query opens both (it sits at their centre)
    nodes = make_nodes([dict(child=[1]), dict(child=[0], depth=1)])
    status, out = run(nodes, leaves(4), nq=nq)
    assert status & B.DEV_ITER_LIMIT
    assert np.isfinite(out).all()  # partial sums are written
    # a node that lists itself
    status, _ = run(make_nodes([dict(child=[0, 0, 0])]), leaves(4), nq=nq)
    assert status & B.DEV_ITER_LIMIT


@pytest.mark.parametrize("nq", [5, 4096])
def test_well_formed_small_tree_raises_nothing(cuda, nq):
    # root with two leaf children holding particles [0, 2) and [2, 4)
    nodes = make_nodes([dict(child=[1, 2], start=0, end=4), dict(depth=1, is_leaf=1, start=0, end=2),
                        dict(depth=1, is_leaf=1, start=2, end=4)])
    status, out = run(nodes, leaves(4), nq=nq)
    assert status == 0
    assert np.isfinite(out).all() and np.abs(out).sum() > 0


@pytest.mark.parametrize("nq", [5, 4096])
def test_child_index_past_the_buffer_sets_bad_bounds(cuda, nq):
    nodes = make_nodes([dict(child=[1, 7]), dict(depth=1, is_leaf=1, start=0, end=2)])
    status, out = run(nodes, leaves(4), nq=nq)
    assert status & B.DEV_BAD_BOUNDS
    assert not status & B.DEV_ITER_LIMIT
    assert np.isfinite(out).all()


@pytest.mark.parametrize("nq", [5, 4096])
def test_leaf_range_past_the_leaf_buffer_sets_bad_bounds(cuda, nq):
    # a leaf that claims particles [0, 9) of a 4-record leaf buffer; the query
    # lies far from it so it is summed particle by particle
    nodes = make_nodes([dict(child=[1]), dict(depth=1, is_leaf=1, start=0, end=9)])
    status, out = run(nodes, leaves(4), nq=nq)
    assert status & B.DEV_BAD_BOUNDS
    assert np.isfinite(out).all()


@pytest.mark.parametrize("nq", [5, 4096])
def test_repeated_children_overflow_the_stack(cuda, nq):
    # 21 nodes, node k lists node k+1 in all eight slots: after v pops the DFS
    # stack holds 1 + 7 v entries and passes its 128 slots at the 19th pop
    specs = [dict(child=[k + 1] * 8, depth=min(k, 10)) for k in range(20)] + [dict(depth=10, is_leaf=1)]
    status, out = run(make_nodes(specs), leaves(4), nq=nq)
    assert status & B.DEV_STACK_OVERFLOW
    assert np.isfinite(out).all()


def test_stochastic_cycles_stop_with_iter_limit(cuda):
    # cycle above the control depth: the subdomain search is bounded
    status, _ = run(make_nodes([dict(child=[1]), dict(child=[0], depth=1)]), leaves(4), stochastic=True)
    assert status & B.DEV_ITER_LIMIT
    # a subdomain node (depth 3) whose children are itself: the sampled
    # descent always continues (the query sits at its centre), so only the
    # 64-level bound ends it
    nodes = make_nodes([dict(child=[1], start=0, end=4), dict(child=[1] * 8, depth=3, start=0, end=4)])
    status, out = run(nodes, leaves(4), stochastic=True)
    assert status & B.DEV_ITER_LIMIT
    assert np.isfinite(out).all()
