"""CPU tests of the C ABI boundary: the library loads, exports every entry
point include/sbh_b200.h declares, reports the reference's byte layouts
(src/sbh_ffi.cu:3949-3963), and rejects invalid arguments on the host before
any device work (no GPU is needed for these paths)."""
import ctypes

import numpy as np
import pytest

import sbh_b200 as B


def test_library_exports_every_declared_symbol():
    lib = B.lib()
    declared = B.header_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared) <= set(B._SIGS), set(declared) - set(B._SIGS)


def test_layout_queries_match_reference():
    assert B.leaf3_size() == 32
    assert B.node3_size() == 4272
    assert B.octree_level3_max_nodes() == 513
    assert B.octree8_node_size() == 104
    assert B.lib().sbh_leaf2_size() == 24
    assert B.lib().sbh_node2_size() == 616
    assert [B._octree8_total_nodes(d) for d in (1, 5, 7)] == [9, 37449, 2396745]


def test_host_validation_without_device():
    L = B.lib()
    null = None
    rc = L.sbh_build_octree8(null, null, null, null, 10, null, null, 0, null, 0, null, 0, null, 0, null, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "max_depth" in B.last_error()
    rc = L.sbh_build_octree8(null, null, null, null, 10, null, null, 3, null, 320, null, 1, null, 0, null, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "node_out size" in B.last_error()
    rc = L.sbh_direct_force_soft(null, null, null, 4, null, 4, null, -1.0, 1.0, 0, 1.0, 256)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "softening" in B.last_error()
    rc = L.sbh_direct_force_soft(null, null, null, 4, null, 4, null, 1e-2, 0.0, 0, 1.0, 256)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "cutoff" in B.last_error()
    rc = L.sbh_direct_force_soft(null, null, null, 4, null, 4, null, 1e-2, 1.0, 0, 1.0, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "threads" in B.last_error()
    rc = L.sbh_barnes_hut_force_octree8(null, null, 33, null, 104, null, 1, null, 2.0, 0, 1.0, 256, null, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "leaf_bytes" in B.last_error()
    rc = L.sbh_barnes_hut_force_octree8_soft(null, null, 32, null, 104, null, 1, null, 2.0, 1e-2, 1.0, 1, -1.0, 0,
                                             1.0, 256, null, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "prune_r_cut_mult" in B.last_error()
    rc = L.sbh_native_build(null, null, null, null, 10, null, 1, 0, 1, null, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "leaf_size" in B.last_error()
    rc = L.sbh_native_build(null, null, null, null, 10, null, 2, 16, 1, null, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "system_offsets" in B.last_error()
    prm = B.NativeParams(2.0, 1e-3, 0.0, 1)
    rc = L.sbh_native_force(null, ctypes.byref(prm), null, ctypes.c_void_p(12345), 1 << 20)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "no native tree" in B.last_error()
    prm = B.NativeTree.params(quadrupole_radius=-1.0)
    rc = L.sbh_native_force(null, ctypes.byref(prm), null, ctypes.c_void_p(12345), 1 << 20)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "quadrupole_radius" in B.last_error()
    prm = B.NativeTree.params(cutoff=0.05, quadrupole=False, prune_radius=0.3, periodic=True, box_length=0.0)
    rc = L.sbh_native_force(null, ctypes.byref(prm), null, ctypes.c_void_p(12345), 1 << 20)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "box_length" in B.last_error()
    rc = L.sbh_barnes_hut_tree(null, 4, 0, null, 0, null, 616, null, 1, null, 2.0, 0.0, 1.0, 0, 1.0, 64, null, 0)
    assert rc == B.SBH_ERR_INVALID_ARGUMENT and "dim" in B.last_error()


def test_workspace_sizes_are_monotone():
    L = B.lib()
    a = L.sbh_build_octree8_workspace_bytes(1000, 5)
    b = L.sbh_build_octree8_workspace_bytes(100000, 5)
    c = L.sbh_build_octree8_workspace_bytes(1000, 7)
    assert 0 < a < b and a < c
    assert L.sbh_build_octree8_workspace_bytes(10, 11) == 0
    n1 = L.sbh_native_workspace_bytes(1 << 20, 1, 16, 0, 1)
    n2 = L.sbh_native_workspace_bytes(1 << 20, 1, 16, 0, 0)
    assert n1 > n2 > 0 and n1 < 1 << 30


def test_python_mirror_validates_like_the_reference():
    # python/jax_sbh_ffi.py raises ValueError before the call; so does the mirror
    with pytest.raises((ValueError, RuntimeError)):
        B.softened_direct_force(np.zeros((4, 2), np.float32), np.zeros(4, np.float32), np.zeros((4, 3), np.float32))
