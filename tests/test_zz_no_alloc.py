"""The octree8 build variant for callers that cannot allocate device memory
at call time (sbh_build_octree8_static): it must give the same buffers as
the ordinary build with a caller workspace, on two calls in a row (the
second call reuses the library's scratch array after the first left its
contents there), and it must refuse sizes beyond its fixed scratch.

Collected last on purpose (file name), so a run that stops at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

import sbh_b200 as B
import sbh_workloads as W

pytestmark = pytest.mark.gpu


def _build(fn_static, dev, p, nrm, m, mn, mx, depth):
    L = B.lib()
    n = p.shape[0]
    total = B._octree8_total_nodes(depth)
    leaf = torch.full((n * 32,), 0xAB, dtype=torch.uint8, device=dev)
    node = torch.full((total * 104,), 0xAB, dtype=torch.uint8, device=dev)
    contrib = torch.full((total * 32,), 0xAB, dtype=torch.uint8, device=dev)
    P, N, M, MN, MX = (torch.as_tensor(a, device=dev) for a in (p, nrm, m, mn, mx))
    s = torch.cuda.current_stream(dev).cuda_stream
    if fn_static:
        rc = L.sbh_build_octree8_static(s, P.data_ptr(), N.data_ptr(), M.data_ptr(), n, MN.data_ptr(), MX.data_ptr(),
                                        depth, leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                        contrib.data_ptr(), contrib.numel())
    else:
        ws = torch.empty(L.sbh_build_octree8_workspace_bytes(n, depth), dtype=torch.uint8, device=dev)
        rc = L.sbh_build_octree8(s, P.data_ptr(), N.data_ptr(), M.data_ptr(), n, MN.data_ptr(), MX.data_ptr(), depth,
                                 leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(), contrib.data_ptr(),
                                 contrib.numel(), ws.data_ptr(), ws.numel())
    assert rc == B.SBH_OK, B.last_error()
    torch.cuda.synchronize()
    return leaf.cpu().numpy(), node.cpu().numpy(), contrib.cpu().numpy()


def test_static_scratch_build_matches_workspace_build_twice(cuda):
    rng = np.random.default_rng(17)
    for call, (n, depth, seed) in enumerate([(50000, 6, 1), (20000, 5, 2)]):
        p, m = W.plummer(n, seed=seed)
        nrm = rng.normal(size=p.shape).astype(np.float32)
        mn = (p.min(0) - np.float32(1e-3)).astype(np.float32)
        mx = (p.max(0) + np.float32(1e-3)).astype(np.float32)
        got = _build(True, cuda, p, nrm, m, mn, mx, depth)
        want = _build(False, cuda, p, nrm, m, mn, mx, depth)
        for g, w, name in zip(got, want, ("leaf", "node", "contrib")):
            np.testing.assert_array_equal(g, w, err_msg=f"call {call}: {name}")


def test_static_scratch_rejects_sizes_beyond_its_limit(cuda):
    L = B.lib()
    limit = L.sbh_build_octree8_static_scratch_bytes()
    assert L.sbh_build_octree8_workspace_bytes(1 << 20, 7) > limit
    rc = L.sbh_build_octree8_static(torch.cuda.current_stream().cuda_stream, None, None, None, 1 << 20, None, None, 7,
                                    None, 0, None, 0, None, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT
    assert "scratch" in B.last_error()
