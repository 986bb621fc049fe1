"""CPU tests of the XLA custom-call handlers (include/sbh_xla_ffi.h): every
handler symbol of the reference (src/sbh_ffi.cu:3580-3947) is exported and
declared, answers XLA's registration-time metadata query with FFI API
version 0.1, and rejects malformed call frames with INVALID_ARGUMENT and the
reference's messages before any device work. The call frames are built by
hand (tests/xla_ffi_emulator.py stands in for the XLA runtime); no GPU, jax
or jaxlib is needed."""
import os
import re

import numpy as np
import pytest

import sbh_b200 as B
from xla_ffi_emulator import DT_F32, DT_S32, DT_U8, ERR_INVALID_ARGUMENT, FakeXla, HandlerError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# every XLA_FFI_DEFINE_HANDLER_SYMBOL of src/sbh_ffi.cu:3580-3947
REFERENCE_HANDLERS = [
    "sbh_bruteforce_gravity_ffi", "sbh_direct_force_soft_ffi", "sbh_direct_force_soft_vjp_ffi",
    "sbh_build_octree_level3_buffers_ffi", "sbh_build_octree8_buffers_ffi", "sbh_barnes_hut_gravity_ffi",
    "sbh_barnes_hut_force_ffi", "sbh_barnes_hut_gravity_ffi_3d", "sbh_barnes_hut_force_ffi_3d",
    "sbh_barnes_hut_force_octree8_ffi", "sbh_barnes_hut_force_octree8_soft_ffi",
    "sbh_barnes_hut_force_octree8_soft_vjp_ffi", "sbh_barnes_hut_force_soft_ffi", "sbh_barnes_hut_force_soft_ffi_3d",
    "sbh_stochastic_bh_gravity_ffi", "sbh_stochastic_bh_gravity_ffi_3d", "sbh_stochastic_bh_force_ffi",
    "sbh_stochastic_bh_force_ffi_3d", "sbh_stochastic_bh_force_octree8_ffi",
    "sbh_stochastic_bh_force_octree8_soft_ffi", "sbh_stochastic_bh_force_octree8_vjp_ffi",
    "sbh_stochastic_bh_force_octree8_soft_vjp_ffi", "sbh_stochastic_bh_force_soft_ffi",
    "sbh_stochastic_bh_force_soft_ffi_3d",
]


def _host_alloc():
    """A runtime allocator returning host memory: the rejections below all
    happen before the scratch is touched."""
    def alloc(size):
        buf = np.zeros(size, np.uint8)
        return buf.ctypes.data, buf
    return alloc


def _f(a):
    a = np.ascontiguousarray(a, np.float32)
    return (DT_F32, a.ctypes.data, a.shape), a


def _u8(n):
    a = np.zeros(n, np.uint8)
    return (DT_U8, a.ctypes.data, a.shape), a


def test_every_reference_handler_is_declared_and_exported():
    text = open(os.path.join(ROOT, "include", "sbh_xla_ffi.h")).read()
    declared = set(re.findall(r"\b(sbh_\w+_ffi(?:_3d)?)\s*\(", text))
    assert declared == set(REFERENCE_HANDLERS)
    lib = B.lib()
    for name in REFERENCE_HANDLERS:
        assert hasattr(lib, name), name


@pytest.mark.parametrize("name", REFERENCE_HANDLERS)
def test_metadata_query_reports_api_version(name):
    assert FakeXla.metadata(getattr(B.lib(), name)) == (0, 1, 0)


def test_non_execute_stage_is_a_no_op():
    x = FakeXla()
    x.call(B.lib().sbh_direct_force_soft_ffi, [], [], {}, stage=0)  # instantiate: nothing decoded


def _direct_call(x, pts=(16, 3), q=(4, 3), out=(4, 3), attrs=None, masses=16, extra_arg=False):
    P, _p = _f(np.zeros(pts))
    M, _m = _f(np.zeros(masses))
    Q, _q = _f(np.zeros(q))
    O, _o = _f(np.zeros(out))
    a = dict(softening_scale=np.float32(1e-2), cutoff_scale=np.float32(1.0), periodic=np.int32(0),
             box_length=np.float32(1.0), threads=np.int32(256))
    a.update(attrs or {})
    args = [P, M, Q] + ([Q] if extra_arg else [])
    x.call(B.lib().sbh_direct_force_soft_ffi, args, [O], a)


@pytest.mark.parametrize("kw,msg", [
    (dict(pts=(16, 2), q=(4, 2), out=(4, 3)), "points/queries must have dim=3"),
    (dict(masses=15), "masses length mismatch"),
    (dict(out=(5, 3)), "out shape mismatch"),
    (dict(attrs=dict(threads=np.int32(0))), "threads must be in [1, 1024]"),
    (dict(attrs=dict(softening_scale=np.float32(-1.0))), "softening_scale must be >= 0"),
    (dict(attrs=dict(cutoff_scale=np.float32(0.0))), "cutoff_scale must be > 0"),
    (dict(extra_arg=True), "Wrong number of arguments"),
    (dict(attrs=dict(threads=np.float32(256))), "Wrong scalar data type"),
])
def test_direct_force_rejects_with_reference_messages(kw, msg):
    x = FakeXla()
    with pytest.raises(HandlerError) as e:
        _direct_call(x, **kw)
    assert e.value.code == ERR_INVALID_ARGUMENT
    assert msg in e.value.message


def test_missing_attribute_and_wrong_dtype_are_reported():
    x = FakeXla()
    P, _p = _f(np.zeros((8, 3)))
    M, _m = _f(np.zeros(8))
    O, _o = _f(np.zeros((4, 3)))
    bad_q = (DT_S32, _p.ctypes.data, (4, 3))
    attrs = dict(softening_scale=np.float32(1e-2), cutoff_scale=np.float32(1.0), periodic=np.int32(0),
                 box_length=np.float32(1.0), threads=np.int32(256))
    with pytest.raises(HandlerError, match="Wrong buffer dtype"):
        x.call(B.lib().sbh_direct_force_soft_ffi, [P, M, bad_q], [O], attrs)
    attrs.pop("threads")
    attrs["thread"] = np.int32(256)
    with pytest.raises(HandlerError, match="missing attribute 'threads'"):
        x.call(B.lib().sbh_direct_force_soft_ffi, [P, M, P], [O], attrs)


@pytest.mark.parametrize("depth,pts,msg", [
    (11, (10, 3), "max_depth must be in [1, 10]"),
    (3, (10, 2), "points must have shape (N, 3)"),
    (3, (10, 3), "node_out size mismatch"),
])
def test_octree8_build_rejects_with_reference_messages(depth, pts, msg):
    x = FakeXla(allocate=_host_alloc())
    P, _p = _f(np.zeros(pts))
    N, _n = _f(np.zeros(pts))
    M, _m = _f(np.zeros(pts[0]))
    C, _c = _f(np.zeros(3))
    leaf, _l = _u8(pts[0] * 32)
    node, _nd = _u8(104)  # not T(3) * 104
    con, _cn = _u8(32)
    with pytest.raises(HandlerError) as e:
        x.call(B.lib().sbh_build_octree8_buffers_ffi, [P, N, M, C, C], [leaf, node, con],
               dict(max_depth=np.int32(depth)))
    assert e.value.code == ERR_INVALID_ARGUMENT and msg in e.value.message
    assert not x.live  # scratch handed back before the handler returned


@pytest.mark.parametrize("name,dim,msg", [
    ("sbh_barnes_hut_force_ffi_3d", 2, "queries dim must be 3"),
    ("sbh_barnes_hut_force_ffi", 3, "queries dim must be 2"),
])
def test_tree_traversals_check_query_dims(name, dim, msg):
    x = FakeXla(allocate=_host_alloc())
    leaf, _l = _u8(32)
    node, _n = _u8(4272)
    Q, _q = _f(np.zeros((4, dim)))
    O, _o = _f(np.zeros((4, dim)))
    with pytest.raises(HandlerError, match=msg):
        x.call(getattr(B.lib(), name), [leaf, node, Q], [O],
               dict(beta=np.float32(2), periodic=np.int32(0), box_length=np.float32(1), threads=np.int32(64)))


def test_octree8_traversal_rejects_bad_buffer_sizes():
    x = FakeXla(allocate=_host_alloc())
    leaf, _l = _u8(33)
    node, _n = _u8(104)
    Q, _q = _f(np.zeros((4, 3)))
    O, _o = _f(np.zeros((4, 3)))
    attrs = dict(beta=np.float32(2), softening_scale=np.float32(1e-2), cutoff_scale=np.float32(1.0),
                 prune_enabled=np.int32(1), prune_r_cut_mult=np.float32(4.0), periodic=np.int32(0),
                 box_length=np.float32(1.0), threads=np.int32(256))
    with pytest.raises(HandlerError, match="leaf_bytes size mismatch"):
        x.call(B.lib().sbh_barnes_hut_force_octree8_soft_ffi, [leaf, node, Q], [O], attrs)
    leaf, _l = _u8(32)
    attrs["prune_r_cut_mult"] = np.float32(-1.0)
    with pytest.raises(HandlerError, match="prune_r_cut_mult must be > 0 when prune_enabled is set"):
        x.call(B.lib().sbh_barnes_hut_force_octree8_soft_ffi, [leaf, node, Q], [O], attrs)
