"""Host side of the sbh_b200 library: ctypes bindings of the C ABI
(``include/sbh_b200.h``) and a torch-tensor mirror of the reference's
``python/jax_sbh_ffi.py`` surface (same function names, keyword defaults,
validation messages and ``custom_vjp`` semantics).

Device memory, streams and autograd come from PyTorch; all arithmetic runs in
the hand-written CUDA kernels of ``libsbh_b200.so``. There is no CPU fallback:
without the built library or without a CUDA device every compute function
raises.
"""
from __future__ import annotations

import ctypes
import os
import re
import threading
from typing import Optional

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsbh_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "sbh_b200.h")
FFI_HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "sbh_xla_ffi.h")

# Target names of the reference FFI (python/jax_sbh_ffi.py:10-34).
TARGETS = {
    "bruteforce_gravity": "sbh_bruteforce_gravity",
    "direct_force_soft": "sbh_direct_force_soft",
    "direct_force_soft_vjp": "sbh_direct_force_soft_vjp",
    "barnes_hut_gravity": "sbh_barnes_hut_gravity",
    "barnes_hut_force": "sbh_barnes_hut_force",
    "barnes_hut_gravity_3d": "sbh_barnes_hut_gravity_3d",
    "barnes_hut_force_3d": "sbh_barnes_hut_force_3d",
    "barnes_hut_force_soft": "sbh_barnes_hut_force_soft",
    "barnes_hut_force_soft_3d": "sbh_barnes_hut_force_soft_3d",
    "stochastic_bh_gravity": "sbh_stochastic_bh_gravity",
    "stochastic_bh_gravity_3d": "sbh_stochastic_bh_gravity_3d",
    "stochastic_bh_force": "sbh_stochastic_bh_force",
    "stochastic_bh_force_3d": "sbh_stochastic_bh_force_3d",
    "stochastic_bh_force_soft": "sbh_stochastic_bh_force_soft",
    "stochastic_bh_force_soft_3d": "sbh_stochastic_bh_force_soft_3d",
    "build_octree_level3_buffers": "sbh_build_octree_level3_buffers",
    "build_octree8_buffers": "sbh_build_octree8_buffers",
    "barnes_hut_force_octree8": "sbh_barnes_hut_force_octree8",
    "barnes_hut_force_octree8_soft": "sbh_barnes_hut_force_octree8_soft",
    "barnes_hut_force_octree8_soft_vjp": "sbh_barnes_hut_force_octree8_soft_vjp",
    "stochastic_bh_force_octree8": "sbh_stochastic_bh_force_octree8",
    "stochastic_bh_force_octree8_soft": "sbh_stochastic_bh_force_octree8_soft",
    "stochastic_bh_force_octree8_vjp": "sbh_stochastic_bh_force_octree8_vjp",
    "stochastic_bh_force_octree8_soft_vjp": "sbh_stochastic_bh_force_octree8_soft_vjp",
}

SBH_OK = 0
SBH_ERR_INVALID_ARGUMENT = 1
SBH_ERR_CUDA = 2
SBH_ERR_WORKSPACE = 3
SBH_ERR_LIMIT = 4
DEV_STACK_OVERFLOW = 0x1
DEV_BAD_BOUNDS = 0x2
DEV_ITER_LIMIT = 0x4


class SbhError(RuntimeError):
    """A CUDA-side failure reported by libsbh_b200 (SBH_ERR_CUDA / _LIMIT)."""


_c_p = ctypes.c_void_p
_c_sz = ctypes.c_size_t
_c_i = ctypes.c_int
_c_i64 = ctypes.c_int64
_c_f = ctypes.c_float
_c_u64 = ctypes.c_uint64

# argtypes of every entry point, keyed by symbol (checked against the header
# by the CPU tests).
_SIGS = {
    "sbh_last_error": ([], ctypes.c_char_p),
    "sbh_version": ([], ctypes.c_char_p),
    "sbh_read_device_status": ([_c_p, _c_p, _c_p], _c_i),
    "sbh_leaf3_size": ([], _c_sz),
    "sbh_node3_size": ([], _c_sz),
    "sbh_octree_level3_max_nodes": ([], _c_sz),
    "sbh_octree8_node_size": ([], _c_sz),
    "sbh_leaf2_size": ([], _c_sz),
    "sbh_node2_size": ([], _c_sz),
    "sbh_octree8_total_nodes": ([_c_i], _c_u64),
    "sbh_traversal_workspace_bytes": ([], _c_sz),
    "sbh_traversal_ordered_workspace_bytes": ([_c_i64], _c_sz),
    "sbh_bruteforce_gravity": ([_c_p, _c_p, _c_p, _c_i64, _c_i, _c_p, _c_i64, _c_p, _c_i, _c_f, _c_i], _c_i),
    "sbh_direct_force_soft": ([_c_p, _c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_f, _c_f, _c_i, _c_f, _c_i], _c_i),
    "sbh_direct_force_soft_vjp": ([_c_p, _c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_p, _c_f, _c_f, _c_i, _c_f, _c_i],
                                  _c_i),
    "sbh_build_octree8_workspace_bytes": ([_c_i64, _c_i], _c_sz),
    "sbh_build_octree8_static_scratch_bytes": ([], _c_sz),
    "sbh_build_octree8_static": ([_c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p,
                                  _c_sz], _c_i),
    "sbh_build_octree8": ([_c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_sz,
                           _c_p, _c_sz], _c_i),
    "sbh_barnes_hut_force_octree8": ([_c_p, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_f, _c_i, _c_f, _c_i,
                                      _c_p, _c_sz], _c_i),
    "sbh_barnes_hut_force_octree8_vjp": ([_c_p, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_p, _c_f, _c_i, _c_f,
                                          _c_i, _c_p, _c_sz], _c_i),
    "sbh_barnes_hut_force_octree8_soft": ([_c_p, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_f, _c_f, _c_f,
                                           _c_i, _c_f, _c_i, _c_f, _c_i, _c_p, _c_sz], _c_i),
    "sbh_barnes_hut_force_octree8_soft_vjp": ([_c_p, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_p, _c_f, _c_f,
                                               _c_f, _c_i, _c_f, _c_i, _c_f, _c_i, _c_p, _c_sz], _c_i),
    "sbh_stochastic_bh_force_octree8": ([_c_p, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_i, _c_i, _c_f,
                                         _c_f, _c_f, _c_i, _c_f, _c_i, _c_f, _c_i, _c_p, _c_sz], _c_i),
    "sbh_stochastic_bh_force_octree8_vjp": ([_c_p, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_p, _c_i,
                                             _c_i, _c_f, _c_f, _c_f, _c_i, _c_f, _c_i, _c_f, _c_i, _c_p, _c_sz], _c_i),
    "sbh_probe_fp32": ([_c_p, _c_p, _c_i, _c_i], _c_i),
    "sbh_probe_fp32x2": ([_c_p, _c_p, _c_i, _c_i], _c_i),
    "sbh_build_octree_level3_workspace_bytes": ([_c_i64], _c_sz),
    "sbh_build_octree_level3": ([_c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_sz, _c_p,
                                 _c_sz], _c_i),
    "sbh_barnes_hut_tree": ([_c_p, _c_i, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_f, _c_f, _c_f, _c_i,
                             _c_f, _c_i, _c_p, _c_sz], _c_i),
    "sbh_barnes_hut_tree_vjp": ([_c_p, _c_i, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_p, _c_f, _c_f,
                                 _c_f, _c_i, _c_f, _c_i, _c_p, _c_sz], _c_i),
    "sbh_stochastic_bh_tree": ([_c_p, _c_i, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_i, _c_i,
                                _c_f, _c_f, _c_i, _c_f, _c_i, _c_p, _c_sz], _c_i),
    "sbh_brute_force_tree": ([_c_p, _c_i, _c_i, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_i], _c_i),
    "sbh_stochastic_bh_tree_shared_seed": ([_c_p, _c_i, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p,
                                            _c_i, _c_i, _c_i, _c_p, _c_sz], _c_i),
    "sbh_stochastic_bh_tree_vjp": ([_c_p, _c_i, _c_i, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_i64, _c_p, _c_p,
                                    _c_i, _c_i, _c_f, _c_f, _c_i, _c_f, _c_i, _c_p, _c_sz], _c_i),
    "sbh_build_quadtree_workspace_bytes": ([_c_i64], _c_sz),
    "sbh_build_adaptive_octree_workspace_bytes": ([_c_i64], _c_sz),
    "sbh_build_adaptive_octree": ([_c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_f, _c_p, _c_sz, _c_p, _c_sz, _c_p,
                                   _c_sz, _c_p, _c_p, _c_sz], _c_i),
    "sbh_build_quadtree": ([_c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_f, _c_p, _c_sz, _c_p, _c_sz, _c_p, _c_sz,
                            _c_p, _c_p, _c_sz], _c_i),
    "sbh_native_group_size": ([], _c_i),
    "sbh_native_release": ([_c_p], _c_i),
    "sbh_native_workspace_bytes": ([_c_i64, _c_i, _c_i, _c_i, _c_i], _c_sz),
    "sbh_native_build": ([_c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_i, _c_i, _c_i, _c_p, _c_sz], _c_i),
    "sbh_native_force": ([_c_p, _c_p, _c_p, _c_p, _c_sz], _c_i),
    "sbh_native_force_vjp": ([_c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_sz], _c_i),
    "sbh_native_adjoint_walk": ([_c_p, _c_p, _c_p, _c_p, _c_p, _c_sz], _c_i),
    "sbh_native_adjoint_finalize": ([_c_p, _c_p, _c_p, _c_p, _c_sz], _c_i),
    "sbh_native_adjoint_query_side": ([_c_p, _c_p, _c_p, _c_sz], _c_i),
    "sbh_native_query_workspace_bytes": ([_c_i64], _c_sz),
    "sbh_native_winding_number": ([_c_p, _c_f, _c_p, _c_i64, _c_p, _c_p, _c_sz, _c_p, _c_sz], _c_i),
    "sbh_native_winding_number_vjp": ([_c_p, _c_f, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_sz, _c_p,
                                       _c_sz], _c_i),
    "sbh_native_stats": ([_c_p, _c_p, _c_sz, _c_p], _c_i),
    "sbh_native_quadrupole_count": ([_c_p, _c_p, _c_sz, _c_p], _c_i),
    "sbh_native_set_group_size": ([_c_p, _c_p, _c_sz, _c_i], _c_i),
    "sbh_native_far_counts": ([_c_p, _c_p, _c_sz, _c_p], _c_i),
    "sbh_native_set_target_range": ([_c_p, _c_p, _c_sz, _c_i64, _c_i64], _c_i),
    "sbh_mesh_sample_workspace_bytes": ([_c_i64], _c_sz),
    "sbh_mesh_vertex_workspace_bytes": ([_c_i64], _c_sz),
    "sbh_mesh_vertex_sources": ([_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_sz], _c_i),
    "sbh_sample_mesh_surface": ([_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_i64, _c_u64, _c_p, _c_p, _c_p, _c_p, _c_sz],
                                _c_i),
    "sbh_native_export": ([_c_p, _c_p, _c_sz, _c_p, _c_p, _c_p, _c_sz, _c_p], _c_i),
    "sbh_native_stochastic_force": ([_c_p, _c_p, _c_f, _c_i, ctypes.c_uint64, _c_p, _c_p, _c_sz], _c_i),
    "sbh_native_stochastic_force_vjp": ([_c_p, _c_p, _c_f, _c_i, ctypes.c_uint64, _c_p, _c_p, _c_p, _c_p, _c_p,
                                         _c_sz], _c_i),
}


class NativeParams(ctypes.Structure):
    """sbh_native_params of include/sbh_b200.h."""

    _fields_ = [("beta", ctypes.c_float), ("softening", ctypes.c_float), ("cutoff", ctypes.c_float),
                ("quadrupole", ctypes.c_int), ("periodic", ctypes.c_int), ("box_length", ctypes.c_float),
                ("prune_radius", ctypes.c_float), ("quadrupole_radius", ctypes.c_float),
                ("quadrupole_linear", ctypes.c_float)]


# Accepted nodes closer to a target group than this many opening radii take
# the quadrupole, farther ones the monopole alone (0: every accepted node
# takes it). With the once-per-group linearized form below the quadrupole of a
# distant node costs little, so every accepted node keeps it.
QUADRUPOLE_RADIUS = 0.0

# Accepted quadrupole nodes with r_g <= QUADRUPOLE_LINEAR |c - cell centre|
# (c the group box centre, r_g its half diagonal) take the quadrupole to first
# order about c, evaluated once per group instead of once per target
# (sbh_native_params.quadrupole_linear; 0: every quadrupole is exact). On the
# bench workload (8 Plummer spheres of 2^20, beta 2, groups of 128) 95% of the
# far interactions are linearized at 0.5; the adjoint walk went from 365 ms
# (exact quadrupole within 1.6 opening radii) to 324 ms at the same force error
# against the FP64 direct sum (2.5e-5).
QUADRUPOLE_LINEAR = 0.5

_lib_handle = None
_lib_lock = threading.Lock()


def library_path() -> str:
    return LIB_PATH


def lib() -> ctypes.CDLL:
    """The loaded libsbh_b200.so (raises if it was not built)."""
    global _lib_handle
    with _lib_lock:
        if _lib_handle is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is not built; run `python barnes-hut_b200/sbh_build.py` "
                                   "(or __graft_entry__.build()) first")
            h = ctypes.CDLL(LIB_PATH)
            for name, (args, res) in _SIGS.items():
                fn = getattr(h, name, None)
                if fn is None:
                    continue
                fn.argtypes = args
                fn.restype = res
            _lib_handle = h
    return _lib_handle


def header_symbols() -> list[str]:
    """Function names declared in include/sbh_b200.h and include/sbh_xla_ffi.h."""
    text = open(HEADER_PATH).read() + open(FFI_HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sbh_[a-z0-9_]+)\s*\(", text)))


def last_error() -> str:
    return lib().sbh_last_error().decode()


def _check(rc: int, what: str) -> None:
    if rc == SBH_OK:
        return
    msg = last_error()
    if rc == SBH_ERR_INVALID_ARGUMENT:
        raise ValueError(f"{what}: {msg}")
    raise SbhError(f"{what}: {msg} (status {rc})")


# ---------------------------------------------------------------------------
# device plumbing
# ---------------------------------------------------------------------------
def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("sbh_b200 needs a CUDA device (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def _stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


_ws_cache: dict = {}


def workspace(nbytes: int, device: Optional[torch.device] = None) -> torch.Tensor:
    """A uint8 device buffer of at least nbytes, reused per (device, stream)."""
    device = device or _device()
    key = (device.index, _stream_ptr(device))
    buf = _ws_cache.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _ws_cache[key] = buf
    return buf


def read_device_status(ws: torch.Tensor) -> int:
    out = ctypes.c_uint32(0)
    _check(lib().sbh_read_device_status(_stream_ptr(ws.device), ws.data_ptr(), ctypes.byref(out)),
           "read_device_status")
    return int(out.value)


def _f32(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float32).contiguous()
    return torch.as_tensor(np.asarray(x, dtype=np.float32), device=device).contiguous()


def _u8(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.uint8).contiguous()
    return torch.as_tensor(np.asarray(x, dtype=np.uint8), device=device).contiguous()


def _p(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


# ---------------------------------------------------------------------------
# layout queries (python/jax_sbh_ffi.py:62-96)
# ---------------------------------------------------------------------------
def leaf3_size() -> int:
    return int(lib().sbh_leaf3_size())


def node3_size() -> int:
    return int(lib().sbh_node3_size())


def octree_level3_max_nodes() -> int:
    return int(lib().sbh_octree_level3_max_nodes())


def octree8_node_size() -> int:
    return int(lib().sbh_octree8_node_size())


def _octree8_total_nodes(max_depth: int) -> int:
    return int(lib().sbh_octree8_total_nodes(int(max_depth)))


# ---------------------------------------------------------------------------
# direct sums (python/jax_sbh_ffi.py:341-480)
# ---------------------------------------------------------------------------
def brute_force_gravity(points, masses, queries, *, periodic: bool = False, box_length: float = 1.0,
                        threads: int = 64) -> torch.Tensor:
    dev = _device()
    points, masses, queries = _f32(points, dev), _f32(masses, dev), _f32(queries, dev)
    if points.ndim != 2 or queries.ndim != 2:
        raise ValueError("points and queries must be rank-2")
    if masses.ndim != 1:
        raise ValueError("masses must be rank-1")
    if points.shape[0] != masses.shape[0]:
        raise ValueError("masses length mismatch")
    if points.shape[1] != queries.shape[1]:
        raise ValueError("dim mismatch")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")
    out = torch.empty(queries.shape[0], dtype=torch.float32, device=dev)
    _check(lib().sbh_bruteforce_gravity(_stream_ptr(dev), _p(points), _p(masses), points.shape[0], points.shape[1],
                                        _p(queries), queries.shape[0], _p(out), int(bool(periodic)),
                                        float(box_length), int(threads)), "brute_force_gravity")
    return out


def _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads):
    if softening_scale < 0:
        raise ValueError("softening_scale must be >= 0")
    if cutoff_scale <= 0:
        raise ValueError("cutoff_scale must be > 0")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")


def softened_direct_force(points, masses, queries, *, softening_scale: float = 1e-2, cutoff_scale: float = 1.0,
                          periodic: bool = False, box_length: float = 1.0, threads: int = 256) -> torch.Tensor:
    dev = _device()
    points, masses, queries = _f32(points, dev), _f32(masses, dev), _f32(queries, dev)
    if points.ndim != 2 or points.shape[1] != 3:
        raise ValueError("points must be (N, 3)")
    if masses.ndim != 1 or masses.shape[0] != points.shape[0]:
        raise ValueError("masses must have shape (N,)")
    if queries.ndim != 2 or queries.shape[1] != 3:
        raise ValueError("queries must be (M, 3)")
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    out = torch.empty((queries.shape[0], 3), dtype=torch.float32, device=dev)
    _check(lib().sbh_direct_force_soft(_stream_ptr(dev), _p(points), _p(masses), points.shape[0], _p(queries),
                                       queries.shape[0], _p(out), float(softening_scale), float(cutoff_scale),
                                       int(bool(periodic)), float(box_length), int(threads)), "softened_direct_force")
    return out


def softened_direct_force_vjp(points, masses, queries, cotangent, *, softening_scale: float = 1e-2,
                              cutoff_scale: float = 1.0, periodic: bool = False, box_length: float = 1.0,
                              threads: int = 256) -> torch.Tensor:
    dev = _device()
    points, masses = _f32(points, dev), _f32(masses, dev)
    queries, cotangent = _f32(queries, dev), _f32(cotangent, dev)
    if points.ndim != 2 or points.shape[1] != 3:
        raise ValueError("points must be (N, 3)")
    if masses.ndim != 1 or masses.shape[0] != points.shape[0]:
        raise ValueError("masses must have shape (N,)")
    if queries.ndim != 2 or queries.shape[1] != 3:
        raise ValueError("queries must be (M, 3)")
    if cotangent.shape != queries.shape:
        raise ValueError("cotangent must have same shape as queries")
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    out = torch.empty((queries.shape[0], 3), dtype=torch.float32, device=dev)
    _check(lib().sbh_direct_force_soft_vjp(_stream_ptr(dev), _p(points), _p(masses), points.shape[0], _p(queries),
                                           queries.shape[0], _p(cotangent), _p(out), float(softening_scale),
                                           float(cutoff_scale), int(bool(periodic)), float(box_length),
                                           int(threads)), "softened_direct_force_vjp")
    return out


class _SoftenedDirectForceRecompute(torch.autograd.Function):
    """custom_vjp of python/jax_sbh_ffi.py:482-594: forward = self-gravity
    direct force, backward = query-side VJP only, grad_masses = 0."""

    @staticmethod
    def forward(ctx, points, masses, softening_scale, cutoff_scale, periodic, box_length, threads):
        ctx.save_for_backward(points, masses)
        ctx.cfg = (softening_scale, cutoff_scale, periodic, box_length, threads)
        return softened_direct_force(points, masses, points, softening_scale=softening_scale,
                                     cutoff_scale=cutoff_scale, periodic=periodic, box_length=box_length,
                                     threads=threads)

    @staticmethod
    def backward(ctx, cot):
        points, masses = ctx.saved_tensors
        s, c, per, box, thr = ctx.cfg
        gp = softened_direct_force_vjp(points, masses, points, cot.contiguous(), softening_scale=s, cutoff_scale=c,
                                       periodic=per, box_length=box, threads=thr)
        return gp, torch.zeros_like(masses), None, None, None, None, None


def softened_direct_force_recompute_vjp(points, masses, *, softening_scale: float = 1e-2, cutoff_scale: float = 1.0,
                                        periodic: bool = False, box_length: float = 1.0,
                                        threads: int = 256) -> torch.Tensor:
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    dev = _device()
    points = points if isinstance(points, torch.Tensor) else _f32(points, dev)
    masses = masses if isinstance(masses, torch.Tensor) else _f32(masses, dev)
    return _SoftenedDirectForceRecompute.apply(points, masses, float(softening_scale), float(cutoff_scale),
                                               bool(periodic), float(box_length), int(threads))


# ---------------------------------------------------------------------------
# octree8 (python/jax_sbh_ffi.py:864-961, 1336-1897)
# ---------------------------------------------------------------------------
def _default_corners(points: torch.Tensor, min_corner, max_corner, dev):
    if min_corner is None:
        min_corner = points.min(dim=0).values - 1e-3
    if max_corner is None:
        max_corner = points.max(dim=0).values + 1e-3
    return _f32(min_corner, dev), _f32(max_corner, dev)


def build_octree8_buffers_with_contrib(points, normals, masses, min_corner=None, max_corner=None, *,
                                       max_depth: int = 7, check_status: bool = True):
    """(leaf_bytes, node_bytes, contrib_bytes) as uint8 device tensors."""
    dev = _device()
    points, normals, masses = _f32(points, dev), _f32(normals, dev), _f32(masses, dev)
    if points.ndim != 2 or points.shape[1] != 3:
        raise ValueError("points must have shape (N, 3)")
    if normals.shape != points.shape:
        raise ValueError("normals shape mismatch")
    if masses.ndim != 1 or masses.shape[0] != points.shape[0]:
        raise ValueError("masses must have shape (N,)")
    if max_depth < 1 or max_depth > 10:
        raise ValueError("max_depth must be in [1, 10]")
    if points.shape[0] == 0 and (min_corner is None or max_corner is None):
        raise ValueError("empty point set needs explicit min_corner/max_corner")
    mn, mx = _default_corners(points, min_corner, max_corner, dev)
    if mn.shape != (3,) or mx.shape != (3,):
        raise ValueError("min_corner/max_corner must have shape (3,)")
    n = points.shape[0]
    total = _octree8_total_nodes(max_depth)
    leaf = torch.empty(n * 32, dtype=torch.uint8, device=dev)
    node = torch.empty(total * 104, dtype=torch.uint8, device=dev)
    contrib = torch.empty(total * 32, dtype=torch.uint8, device=dev)
    need = int(lib().sbh_build_octree8_workspace_bytes(n, int(max_depth)))
    ws = workspace(need, dev)
    _check(lib().sbh_build_octree8(_stream_ptr(dev), _p(points), _p(normals), _p(masses), n, _p(mn), _p(mx),
                                   int(max_depth), _p(leaf), leaf.numel(), _p(node), node.numel(), _p(contrib),
                                   contrib.numel(), _p(ws), ws.numel()), "build_octree8_buffers")
    if check_status:
        st = read_device_status(ws)
        if st & DEV_BAD_BOUNDS:
            raise ValueError("invalid bounds span")
    return leaf, node, contrib


def build_octree8_buffers(points, normals, masses, min_corner=None, max_corner=None, *, max_depth: int = 7):
    leaf, node, _ = build_octree8_buffers_with_contrib(points, normals, masses, min_corner, max_corner,
                                                       max_depth=max_depth)
    return leaf, node


def _check_traversal(queries, periodic, box_length, threads):
    if queries.ndim != 2 or queries.shape[1] != 3:
        raise ValueError("queries must be (M, 3)")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")


def _status_after(ws, what, check_status):
    if check_status:
        st = read_device_status(ws)
        if st & (DEV_STACK_OVERFLOW | DEV_ITER_LIMIT):
            raise SbhError(f"{what}: device traversal limit reached (status 0x{st:x})")


def _octree8_ws_bytes(nq: int) -> int:
    """Workspace with room to take the queries in Morton order, which lets a
    warp walk 32 neighbouring queries down one shared stack (the results do
    not depend on the order)."""
    return int(lib().sbh_traversal_ordered_workspace_bytes(int(nq)))


def barnes_hut_force_octree8(leaf_bytes, node_bytes, queries, *, beta: float = 2.0, periodic: bool = False,
                             box_length: float = 1.0, threads: int = 256, check_status: bool = False):
    dev = _device()
    leaf, node, queries = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _f32(queries, dev)
    _check_traversal(queries, periodic, box_length, threads)
    out = torch.empty((queries.shape[0], 3), dtype=torch.float32, device=dev)
    ws = workspace(_octree8_ws_bytes(queries.shape[0]), dev)
    _check(lib().sbh_barnes_hut_force_octree8(_stream_ptr(dev), _p(leaf), leaf.numel(), _p(node), node.numel(),
                                              _p(queries), queries.shape[0], _p(out), float(beta), int(bool(periodic)),
                                              float(box_length), int(threads), _p(ws), ws.numel()),
           "barnes_hut_force_octree8")
    _status_after(ws, "barnes_hut_force_octree8", check_status)
    return out


def barnes_hut_force_octree8_vjp(leaf_bytes, node_bytes, queries, cotangent, *, beta: float = 2.0,
                                 periodic: bool = False, box_length: float = 1.0, threads: int = 256,
                                 check_status: bool = False):
    """Analytic query-side VJP of barnes_hut_force_octree8 (the reference's
    function of this name takes central finite differences of the forward,
    python/jax_sbh_ffi.py:1372-1395)."""
    dev = _device()
    leaf, node, queries = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _f32(queries, dev)
    cot = _f32(cotangent, dev)
    _check_traversal(queries, periodic, box_length, threads)
    if cot.shape != queries.shape:
        raise ValueError("cotangent must have same shape as queries")
    out = torch.empty((queries.shape[0], 3), dtype=torch.float32, device=dev)
    ws = workspace(_octree8_ws_bytes(queries.shape[0]), dev)
    _check(lib().sbh_barnes_hut_force_octree8_vjp(_stream_ptr(dev), _p(leaf), leaf.numel(), _p(node), node.numel(),
                                                  _p(queries), queries.shape[0], _p(cot), _p(out), float(beta),
                                                  int(bool(periodic)), float(box_length), int(threads), _p(ws),
                                                  ws.numel()), "barnes_hut_force_octree8_vjp")
    _status_after(ws, "barnes_hut_force_octree8_vjp", check_status)
    return out


def softened_barnes_hut_force_octree8(leaf_bytes, node_bytes, queries, *, beta: float = 2.0,
                                      softening_scale: float = 1e-2, cutoff_scale: float = 1.0,
                                      prune_enabled: bool = True, prune_r_cut_mult: float = 4.0,
                                      periodic: bool = False, box_length: float = 1.0, threads: int = 256,
                                      check_status: bool = False):
    dev = _device()
    leaf, node, queries = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _f32(queries, dev)
    _check_traversal(queries, periodic, box_length, threads)
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    if prune_enabled and prune_r_cut_mult <= 0:
        raise ValueError("prune_r_cut_mult must be > 0 when prune_enabled=True")
    out = torch.empty((queries.shape[0], 3), dtype=torch.float32, device=dev)
    ws = workspace(_octree8_ws_bytes(queries.shape[0]), dev)
    _check(lib().sbh_barnes_hut_force_octree8_soft(
        _stream_ptr(dev), _p(leaf), leaf.numel(), _p(node), node.numel(), _p(queries), queries.shape[0], _p(out),
        float(beta), float(softening_scale), float(cutoff_scale), int(bool(prune_enabled)), float(prune_r_cut_mult),
        int(bool(periodic)), float(box_length), int(threads), _p(ws), ws.numel()), "softened_barnes_hut_force_octree8")
    _status_after(ws, "softened_barnes_hut_force_octree8", check_status)
    return out


def softened_barnes_hut_force_octree8_vjp(leaf_bytes, node_bytes, queries, cotangent, *, beta: float = 2.0,
                                          softening_scale: float = 1e-2, cutoff_scale: float = 1.0,
                                          prune_enabled: bool = True, prune_r_cut_mult: float = 4.0,
                                          periodic: bool = False, box_length: float = 1.0, threads: int = 256,
                                          check_status: bool = False):
    dev = _device()
    leaf, node = _u8(leaf_bytes, dev), _u8(node_bytes, dev)
    queries, cotangent = _f32(queries, dev), _f32(cotangent, dev)
    _check_traversal(queries, periodic, box_length, threads)
    if cotangent.shape != queries.shape:
        raise ValueError("cotangent must have same shape as queries")
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    if prune_enabled and prune_r_cut_mult <= 0:
        raise ValueError("prune_r_cut_mult must be > 0 when prune_enabled=True")
    out = torch.empty((queries.shape[0], 3), dtype=torch.float32, device=dev)
    ws = workspace(_octree8_ws_bytes(queries.shape[0]), dev)
    _check(lib().sbh_barnes_hut_force_octree8_soft_vjp(
        _stream_ptr(dev), _p(leaf), leaf.numel(), _p(node), node.numel(), _p(queries), queries.shape[0],
        _p(cotangent), _p(out), float(beta), float(softening_scale), float(cutoff_scale), int(bool(prune_enabled)),
        float(prune_r_cut_mult), int(bool(periodic)), float(box_length), int(threads), _p(ws), ws.numel()),
        "softened_barnes_hut_force_octree8_vjp")
    _status_after(ws, "softened_barnes_hut_force_octree8_vjp", check_status)
    return out


def _stochastic_octree8(vjp, softened, leaf_bytes, node_bytes, queries, cotangent, beta, samples_per_subdomain,
                        seed, softening_scale, cutoff_scale, prune_enabled, prune_r_cut_mult, periodic, box_length,
                        threads, check_status):
    dev = _device()
    leaf, node, queries = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _f32(queries, dev)
    _check_traversal(queries, periodic, box_length, threads)
    if softened:
        _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
        if prune_enabled and prune_r_cut_mult <= 0:
            raise ValueError("prune_r_cut_mult must be > 0 when prune_enabled=True")
    out = torch.empty((queries.shape[0], 3), dtype=torch.float32, device=dev)
    ws = workspace(_octree8_ws_bytes(queries.shape[0]), dev)
    common = (float(beta), float(softening_scale), float(cutoff_scale), int(bool(prune_enabled)),
              float(prune_r_cut_mult), int(bool(periodic)), float(box_length), int(threads), _p(ws), ws.numel())
    if vjp:
        cot = _f32(cotangent, dev)
        if cot.shape != queries.shape:
            raise ValueError("cotangent must have same shape as queries")
        rc = lib().sbh_stochastic_bh_force_octree8_vjp(_stream_ptr(dev), int(softened), _p(leaf), leaf.numel(),
                                                       _p(node), node.numel(), _p(queries), queries.shape[0], _p(cot),
                                                       _p(out), int(samples_per_subdomain), int(seed), *common)
    else:
        rc = lib().sbh_stochastic_bh_force_octree8(_stream_ptr(dev), int(softened), _p(leaf), leaf.numel(), _p(node),
                                                   node.numel(), _p(queries), queries.shape[0], _p(out),
                                                   int(samples_per_subdomain), int(seed), *common)
    _check(rc, "stochastic_barnes_hut_force_octree8")
    _status_after(ws, "stochastic_barnes_hut_force_octree8", check_status)
    return out


def stochastic_barnes_hut_force_octree8(leaf_bytes, node_bytes, queries, *, beta: float = 1.0,
                                        samples_per_subdomain: int = 1, seed: int = 0, periodic: bool = False,
                                        box_length: float = 1.0, threads: int = 256, check_status: bool = False):
    return _stochastic_octree8(False, False, leaf_bytes, node_bytes, queries, None, beta, samples_per_subdomain,
                               seed, 0.0, 1.0, False, 4.0, periodic, box_length, threads, check_status)


def stochastic_barnes_hut_force_octree8_vjp(leaf_bytes, node_bytes, queries, cotangent, *, beta: float = 1.0,
                                            samples_per_subdomain: int = 1, seed: int = 0, periodic: bool = False,
                                            box_length: float = 1.0, threads: int = 256,
                                            check_status: bool = False):
    """Analytic query-side VJP kernel (the reference's Python wrapper of the same
    name differentiates by finite differences, python/jax_sbh_ffi.py:1490-1535)."""
    return _stochastic_octree8(True, False, leaf_bytes, node_bytes, queries, cotangent, beta, samples_per_subdomain,
                               seed, 0.0, 1.0, False, 4.0, periodic, box_length, threads, check_status)


def softened_stochastic_barnes_hut_force_octree8(leaf_bytes, node_bytes, queries, *, beta: float = 1.0,
                                                 samples_per_subdomain: int = 1, seed: int = 0,
                                                 softening_scale: float = 1e-2, cutoff_scale: float = 1.0,
                                                 prune_enabled: bool = True, prune_r_cut_mult: float = 4.0,
                                                 periodic: bool = False, box_length: float = 1.0, threads: int = 256,
                                                 check_status: bool = False):
    return _stochastic_octree8(False, True, leaf_bytes, node_bytes, queries, None, beta, samples_per_subdomain, seed,
                               softening_scale, cutoff_scale, prune_enabled, prune_r_cut_mult, periodic, box_length,
                               threads, check_status)


def softened_stochastic_barnes_hut_force_octree8_vjp(leaf_bytes, node_bytes, queries, cotangent, *,
                                                     beta: float = 1.0, samples_per_subdomain: int = 1, seed: int = 0,
                                                     softening_scale: float = 1e-2, cutoff_scale: float = 1.0,
                                                     prune_enabled: bool = True, prune_r_cut_mult: float = 4.0,
                                                     periodic: bool = False, box_length: float = 1.0,
                                                     threads: int = 256, use_ffi: bool = True,
                                                     check_status: bool = False):
    """Analytic query-side VJP. The reference defaults to use_ffi=False, an
    element-wise finite difference with 6*M forward calls
    (python/jax_sbh_ffi.py:1591-1628); here both settings run the kernel."""
    del use_ffi
    return _stochastic_octree8(True, True, leaf_bytes, node_bytes, queries, cotangent, beta, samples_per_subdomain,
                               seed, softening_scale, cutoff_scale, prune_enabled, prune_r_cut_mult, periodic,
                               box_length, threads, check_status)


class _SoftenedOctree8Recompute(torch.autograd.Function):
    """custom_vjp of python/jax_sbh_ffi.py:1731-1897: forward builds the tree
    and evaluates self-gravity; backward rebuilds the tree from the saved
    inputs and applies the query-side VJP; grad_masses = 0."""

    @staticmethod
    def forward(ctx, points, masses, cfg):
        ctx.save_for_backward(points, masses)
        ctx.cfg = cfg
        return _octree8_self_force(points, masses, cfg)

    @staticmethod
    def backward(ctx, cot):
        points, masses = ctx.saved_tensors
        beta, s, c, depth, prune, mult, per, box, thr = ctx.cfg
        leaf, node = build_octree8_buffers(points, torch.zeros_like(points), masses, max_depth=depth)
        gp = softened_barnes_hut_force_octree8_vjp(leaf, node, points, cot.contiguous(), beta=beta,
                                                   softening_scale=s, cutoff_scale=c, prune_enabled=prune,
                                                   prune_r_cut_mult=mult, periodic=per, box_length=box,
                                                   threads=thr)
        return gp, torch.zeros_like(masses), None


def _octree8_self_force(points, masses, cfg):
    beta, s, c, depth, prune, mult, per, box, thr = cfg
    leaf, node = build_octree8_buffers(points, torch.zeros_like(points), masses, max_depth=depth)
    return softened_barnes_hut_force_octree8(leaf, node, points, beta=beta, softening_scale=s, cutoff_scale=c,
                                             prune_enabled=prune, prune_r_cut_mult=mult, periodic=per,
                                             box_length=box, threads=thr)


def softened_barnes_hut_force_octree8_recompute_vjp(points, masses, *, beta: float = 2.0,
                                                    softening_scale: float = 1e-2, cutoff_scale: float = 1.0,
                                                    max_depth: int = 7, prune_enabled: bool = True,
                                                    prune_r_cut_mult: float = 4.0, periodic: bool = False,
                                                    box_length: float = 1.0, threads: int = 256) -> torch.Tensor:
    if prune_enabled and prune_r_cut_mult <= 0:
        raise ValueError("prune_r_cut_mult must be > 0 when prune_enabled=True")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")
    dev = _device()
    points = points if isinstance(points, torch.Tensor) else _f32(points, dev)
    masses = masses if isinstance(masses, torch.Tensor) else _f32(masses, dev)
    cfg = (float(beta), float(softening_scale), float(cutoff_scale), int(max_depth), bool(prune_enabled),
           float(prune_r_cut_mult), bool(periodic), float(box_length), int(threads))
    return _SoftenedOctree8Recompute.apply(points, masses, cfg)


class _StochasticOctree8Recompute(torch.autograd.Function):
    """custom_vjp of python/jax_sbh_ffi.py:1900-2046 (softened variant
    :2049-2248): forward builds the tree and evaluates the stochastic
    estimate at the points themselves; backward rebuilds the tree from the
    saved inputs and applies the query-side VJP with the same seed;
    grad_masses = 0."""

    @staticmethod
    def forward(ctx, points, masses, softened, cfg):
        ctx.save_for_backward(points, masses)
        ctx.softened, ctx.cfg = softened, cfg
        return _stochastic_octree8_self(False, softened, points, masses, None, cfg)

    @staticmethod
    def backward(ctx, cot):
        points, masses = ctx.saved_tensors
        gp = _stochastic_octree8_self(True, ctx.softened, points, masses, cot.contiguous(), ctx.cfg)
        return gp, torch.zeros_like(masses), None, None


def _stochastic_octree8_self(vjp, softened, points, masses, cot, cfg):
    beta, sps, seed, s, c, depth, prune, mult, per, box, thr = cfg
    leaf, node = build_octree8_buffers(points, torch.zeros_like(points), masses, max_depth=depth)
    return _stochastic_octree8(vjp, softened, leaf, node, points, cot, beta, sps, seed, s, c, prune, mult, per, box,
                               thr, False)


def stochastic_barnes_hut_force_octree8_recompute_vjp(points, masses, *, beta: float = 1.0,
                                                      samples_per_subdomain: int = 1, seed: int = 0,
                                                      max_depth: int = 7, periodic: bool = False,
                                                      box_length: float = 1.0, threads: int = 256) -> torch.Tensor:
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")
    dev = _device()
    points = points if isinstance(points, torch.Tensor) else _f32(points, dev)
    masses = masses if isinstance(masses, torch.Tensor) else _f32(masses, dev)
    cfg = (float(beta), int(samples_per_subdomain), int(seed), 0.0, 1.0, int(max_depth), False, 4.0, bool(periodic),
           float(box_length), int(threads))
    return _StochasticOctree8Recompute.apply(points, masses, False, cfg)


def softened_stochastic_barnes_hut_force_octree8_recompute_vjp(points, masses, *, beta: float = 1.0,
                                                               samples_per_subdomain: int = 1, seed: int = 0,
                                                               softening_scale: float = 1e-2,
                                                               cutoff_scale: float = 1.0, max_depth: int = 7,
                                                               prune_enabled: bool = True,
                                                               prune_r_cut_mult: float = 4.0, periodic: bool = False,
                                                               box_length: float = 1.0,
                                                               threads: int = 256) -> torch.Tensor:
    if prune_enabled and prune_r_cut_mult <= 0:
        raise ValueError("prune_r_cut_mult must be > 0 when prune_enabled=True")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")
    dev = _device()
    points = points if isinstance(points, torch.Tensor) else _f32(points, dev)
    masses = masses if isinstance(masses, torch.Tensor) else _f32(masses, dev)
    cfg = (float(beta), int(samples_per_subdomain), int(seed), float(softening_scale), float(cutoff_scale),
           int(max_depth), bool(prune_enabled), float(prune_r_cut_mult), bool(periodic), float(box_length),
           int(threads))
    return _StochasticOctree8Recompute.apply(points, masses, True, cfg)


# register_* (python/jax_sbh_ffi.py:99-338): hand this library's XLA
# handlers (include/sbh_xla_ffi.h, the reference's symbol names) to XLA under
# the reference's target names. With jax importable they register exactly as
# the reference does (jax.ffi.pycapsule, platform "CUDA", api_version 1);
# without jax there is no XLA to register with, and the torch functions of
# this module call the same kernels through the C entry points.
_FFI_TARGETS = {
    "register_bruteforce_gravity": [("sbh_bruteforce_gravity", "sbh_bruteforce_gravity_ffi")],
    "register_softened_direct_force": [("sbh_direct_force_soft", "sbh_direct_force_soft_ffi")],
    "register_softened_direct_force_vjp": [("sbh_direct_force_soft_vjp", "sbh_direct_force_soft_vjp_ffi")],
    "register_build_octree_level3_buffers": [("sbh_build_octree_level3_buffers",
                                              "sbh_build_octree_level3_buffers_ffi")],
    "register_build_octree8_buffers": [("sbh_build_octree8_buffers", "sbh_build_octree8_buffers_ffi")],
    "register_barnes_hut_gravity": [("sbh_barnes_hut_gravity", "sbh_barnes_hut_gravity_ffi"),
                                    ("sbh_barnes_hut_gravity_3d", "sbh_barnes_hut_gravity_ffi_3d")],
    "register_stochastic_barnes_hut_gravity": [("sbh_stochastic_bh_gravity", "sbh_stochastic_bh_gravity_ffi"),
                                               ("sbh_stochastic_bh_gravity_3d", "sbh_stochastic_bh_gravity_ffi_3d")],
    "register_stochastic_barnes_hut_force": [("sbh_stochastic_bh_force", "sbh_stochastic_bh_force_ffi"),
                                             ("sbh_stochastic_bh_force_3d", "sbh_stochastic_bh_force_ffi_3d")],
    "register_softened_stochastic_barnes_hut_force": [
        ("sbh_stochastic_bh_force_soft", "sbh_stochastic_bh_force_soft_ffi"),
        ("sbh_stochastic_bh_force_soft_3d", "sbh_stochastic_bh_force_soft_ffi_3d")],
    "register_barnes_hut_force": [("sbh_barnes_hut_force", "sbh_barnes_hut_force_ffi"),
                                  ("sbh_barnes_hut_force_3d", "sbh_barnes_hut_force_ffi_3d")],
    "register_softened_barnes_hut_force": [("sbh_barnes_hut_force_soft", "sbh_barnes_hut_force_soft_ffi"),
                                           ("sbh_barnes_hut_force_soft_3d", "sbh_barnes_hut_force_soft_ffi_3d")],
    "register_barnes_hut_force_octree8": [("sbh_barnes_hut_force_octree8", "sbh_barnes_hut_force_octree8_ffi")],
    "register_softened_barnes_hut_force_octree8": [("sbh_barnes_hut_force_octree8_soft",
                                                    "sbh_barnes_hut_force_octree8_soft_ffi")],
    "register_softened_barnes_hut_force_octree8_vjp": [("sbh_barnes_hut_force_octree8_soft_vjp",
                                                        "sbh_barnes_hut_force_octree8_soft_vjp_ffi")],
    "register_stochastic_barnes_hut_force_octree8": [("sbh_stochastic_bh_force_octree8",
                                                      "sbh_stochastic_bh_force_octree8_ffi")],
    "register_softened_stochastic_barnes_hut_force_octree8": [("sbh_stochastic_bh_force_octree8_soft",
                                                               "sbh_stochastic_bh_force_octree8_soft_ffi")],
    "register_stochastic_barnes_hut_force_octree8_vjp": [("sbh_stochastic_bh_force_octree8_vjp",
                                                          "sbh_stochastic_bh_force_octree8_vjp_ffi")],
    "register_softened_stochastic_barnes_hut_force_octree8_vjp": [("sbh_stochastic_bh_force_octree8_soft_vjp",
                                                                   "sbh_stochastic_bh_force_octree8_soft_vjp_ffi")],
}


# the handlers' C signature: XLA_FFI_Error* handler(XLA_FFI_CallFrame*)
for _pairs in _FFI_TARGETS.values():
    for _target, _symbol in _pairs:
        _SIGS[_symbol] = ([_c_p], _c_p)


def _make_register(pairs):
    def register(path: Optional[str] = None) -> None:
        """Registers this library's XLA handlers for the reference's target
        names when jax is importable (the reference's call, api_version 1);
        otherwise only loads the library. `path` is accepted for the
        reference's signature; this module always uses its in-tree build."""
        handle = lib()
        try:
            import jax  # noqa: F401  (optional: only needed to hand the handlers to XLA)
        except ImportError:
            return
        for target, symbol in pairs:
            jax.ffi.register_ffi_target(target, jax.ffi.pycapsule(getattr(handle, symbol)), platform="CUDA",
                                        api_version=1)
    return register


for _name, _pairs in _FFI_TARGETS.items():
    globals()[_name] = _make_register(_pairs)


# ---------------------------------------------------------------------------
# mesh surface sampling (python/old_interface/sampler.py:45-78,
# python/old_interface/source.py:119-155)
# ---------------------------------------------------------------------------
def sample_points_on_mesh(num_particles: int, V, F, *, seed: int = 0, device=None):
    """(points (n, 3), normals (n, 3), weights (n,)) on the device: points
    uniform on the surface of the triangle mesh (V: (nv, 3) vertices, F:
    (nf, 3) vertex indices), each with its face's unit normal e1 x e2 / |e1 x
    e2| and the weight total area / n. Same distribution as the reference's
    sample_points_on_mesh; the stream is the counter-based splitmix64 of
    sbh_sample_mesh_surface, so (seed, sample index) fixes every sample.
    Raises SbhError when a face references a missing vertex or the mesh has
    no area (read back from the device status word, which synchronises)."""
    device = device or (V.device if isinstance(V, torch.Tensor) and V.is_cuda else _device())
    v = _f32(V, device)
    f = F.to(device=device, dtype=torch.int32).contiguous() if isinstance(F, torch.Tensor) else \
        torch.as_tensor(np.asarray(F, dtype=np.int32), device=device).contiguous()
    if v.ndim != 2 or v.shape[1] != 3 or f.ndim != 2 or f.shape[1] != 3:
        raise ValueError("V must be (nv, 3) and F (nf, 3)")
    n = int(num_particles)
    if n < 0:
        raise ValueError("num_particles must be >= 0")
    pts = torch.empty((n, 3), dtype=torch.float32, device=device)
    nrm = torch.empty((n, 3), dtype=torch.float32, device=device)
    w = torch.empty(n, dtype=torch.float32, device=device)
    ws = workspace(int(lib().sbh_mesh_sample_workspace_bytes(f.shape[0])), device)
    _check(lib().sbh_sample_mesh_surface(_stream_ptr(device), _p(v), v.shape[0], _p(f), f.shape[0], n,
                                         int(seed) & 0xFFFFFFFFFFFFFFFF, _p(pts), _p(nrm), _p(w), _p(ws),
                                         ws.numel()), "sample_mesh_surface")
    if n > 0 and read_device_status(ws) & DEV_BAD_BOUNDS:
        raise SbhError("sample_mesh_surface: a face references a missing vertex, or the mesh has no area")
    return pts, nrm, w


class MeshSurface:
    """Winding-number sources sampled on a triangle mesh (the reference's
    MeshSurface source, python/old_interface/source.py:119-155): the mesh is
    centred and scaled so its largest extent is `scale`, then sample() draws
    points, face normals and area weights on the device."""

    def __init__(self, V, F, scale: float = 1.0, device=None):
        V = np.asarray(V.cpu() if isinstance(V, torch.Tensor) else V, dtype=np.float64)
        vmin, vmax = V.min(axis=0), V.max(axis=0)
        width = float(np.max(vmax - vmin))
        if not width > 0:
            raise ValueError("the mesh has zero extent")
        self.V = ((V - (vmax + vmin) / 2) / width * scale).astype(np.float32)
        self.F = np.asarray(F.cpu() if isinstance(F, torch.Tensor) else F, dtype=np.int32)
        self.device = device

    def sample(self, num_points: int, seed: int = 0):
        return sample_points_on_mesh(num_points, self.V, self.F, seed=seed, device=self.device)


def mesh_vertex_sources(V, F, *, device=None):
    """(points (nv, 3), normals (nv, 3), masses (nv,)) on the device: every
    vertex of the triangle mesh as a winding-number source, with the
    area-weighted vertex normal (igl.per_vertex_normals(V, F, 1)) and the
    mixed Voronoi area (the diagonal of igl.massmatrix's default Voronoi mass
    matrix) as its mass; the masses sum to the surface area. Raises SbhError
    when a face references a missing vertex (read back from the device status
    word, which synchronises)."""
    device = device or (V.device if isinstance(V, torch.Tensor) and V.is_cuda else _device())
    v = _f32(V, device)
    f = F.to(device=device, dtype=torch.int32).contiguous() if isinstance(F, torch.Tensor) else \
        torch.as_tensor(np.asarray(F, dtype=np.int32), device=device).contiguous()
    if v.ndim != 2 or v.shape[1] != 3 or f.ndim != 2 or f.shape[1] != 3:
        raise ValueError("V must be (nv, 3) and F (nf, 3)")
    nv = v.shape[0]
    nrm = torch.empty((nv, 3), dtype=torch.float32, device=device)
    m = torch.empty(nv, dtype=torch.float32, device=device)
    ws = workspace(int(lib().sbh_mesh_vertex_workspace_bytes(nv)), device)
    _check(lib().sbh_mesh_vertex_sources(_stream_ptr(device), _p(v), nv, _p(f), f.shape[0], _p(nrm), _p(m), _p(ws),
                                         ws.numel()), "mesh_vertex_sources")
    if nv > 0 and read_device_status(ws) & DEV_BAD_BOUNDS:
        raise SbhError("mesh_vertex_sources: a face references a missing vertex")
    return v, nrm, m


class MeshVertices:
    """Winding-number sources at the vertices of a triangle mesh (the
    reference's MeshVertices source, python/old_interface/source.py:85-115):
    the mesh is centred and scaled so its largest extent is `scale`; sample()
    returns the vertices, their area-weighted normals and their Voronoi
    masses (the reference ignores the requested count, and so does this)."""

    def __init__(self, V, F, scale: float = 1.0, device=None):
        V = np.asarray(V.cpu() if isinstance(V, torch.Tensor) else V, dtype=np.float64)
        vmin, vmax = V.min(axis=0), V.max(axis=0)
        width = float(np.max(vmax - vmin))
        if not width > 0:
            raise ValueError("the mesh has zero extent")
        self.V = ((V - (vmax + vmin) / 2) / width * scale).astype(np.float32)
        self.F = np.asarray(F.cpu() if isinstance(F, torch.Tensor) else F, dtype=np.int32)
        self.device = device

    def sample(self, num_points: int = 0):
        return mesh_vertex_sources(self.V, self.F, device=self.device)


# ---------------------------------------------------------------------------
# native adaptive octree (new entry points; no reference counterpart)
# ---------------------------------------------------------------------------
def native_group_size() -> int:
    """Most targets in one walk group of the native tree."""
    return int(lib().sbh_native_group_size())


class NativeTree:
    """A native tree (or forest of independent systems) living in a device
    workspace. build() once, then force(), force_vjp() and
    winding_number() evaluate it; the workspace is reused across builds of
    the same size."""

    NODE_BYTES = 80

    def __init__(self, device=None):
        self.device = device or _device()
        self.ws = None
        self.qws = None
        self.n = 0
        self.num_systems = 1
        self.leaf_size = 16
        self.normals = False
        self.adjoint = False

    def build(self, points, masses, normals=None, system_offsets=None, *, leaf_size: int = 16,
              with_adjoint: bool = True, group_size: Optional[int] = None):
        """Builds the tree (or forest) into this object's workspace.
        group_size: most targets per walk group (default native_group_size();
        32 suits walks bounded by a prune radius)."""
        if group_size is not None and not 1 <= int(group_size) <= native_group_size():
            raise ValueError(f"group_size must be in [1, {native_group_size()}]")
        dev = self.device
        points, masses = _f32(points, dev), _f32(masses, dev)
        if points.ndim != 2 or points.shape[1] != 3:
            raise ValueError("points must have shape (N, 3)")
        if masses.ndim != 1 or masses.shape[0] != points.shape[0]:
            raise ValueError("masses must have shape (N,)")
        nrm = None
        if normals is not None:
            nrm = _f32(normals, dev)
            if nrm.shape != points.shape:
                raise ValueError("normals shape mismatch")
        if not 1 <= leaf_size <= 32:
            raise ValueError("leaf_size must be in [1, 32]")
        offs = None
        nsys = 1
        if system_offsets is not None:
            offs = torch.as_tensor(np.asarray(system_offsets, dtype=np.int64), device=dev) \
                if not isinstance(system_offsets, torch.Tensor) else system_offsets.to(dev, torch.int64)
            nsys = int(offs.numel()) - 1
            if nsys < 1:
                raise ValueError("system_offsets needs at least two entries")
        n = points.shape[0]
        need = int(lib().sbh_native_workspace_bytes(n, nsys, int(leaf_size), int(nrm is not None), int(with_adjoint)))
        if self.ws is None or self.ws.numel() < need:
            self.release()
            self.ws = torch.empty(need, dtype=torch.uint8, device=dev)
        self._keep = (points, masses, nrm, offs)
        _check(lib().sbh_native_build(_stream_ptr(dev), _p(points), _p(masses), _p(nrm), n, _p(offs), nsys,
                                      int(leaf_size), int(with_adjoint), _p(self.ws), self.ws.numel()),
               "native_build")
        self.n, self.num_systems, self.leaf_size = n, nsys, int(leaf_size)
        self.normals, self.adjoint = nrm is not None, bool(with_adjoint)
        if group_size is not None and int(group_size) != native_group_size():
            self.set_group_size(int(group_size))
        return self

    def release(self) -> None:
        """Drops this tree's entry in the library's host registry (before the
        workspace memory goes back to the allocator, which may hand the same
        address to another tree)."""
        if self.ws is not None:
            lib().sbh_native_release(_p(self.ws))

    def __del__(self):
        try:
            self.release()
        except Exception:  # interpreter shutdown: the library may be gone
            pass

    def set_target_range(self, begin: int, end: int) -> None:
        """Walk only the target groups starting at sorted positions
        [begin, end); other targets' force rows are zero and the gradients
        are this share's partial sums (sbh_native_set_target_range)."""
        _check(lib().sbh_native_set_target_range(_stream_ptr(self.device), _p(self.ws), self.ws.numel(),
                                                 int(begin), int(end)), "native_set_target_range")

    def set_group_size(self, group_size: int) -> None:
        """Re-cuts the target groups with at most group_size targets each."""
        _check(lib().sbh_native_set_group_size(_stream_ptr(self.device), _p(self.ws), self.ws.numel(),
                                               int(group_size)), "native_set_group_size")

    @staticmethod
    def params(beta=2.0, softening=1e-3, cutoff=0.0, quadrupole=True, periodic=False, box_length=1.0,
               prune_radius=0.0, quadrupole_radius=QUADRUPOLE_RADIUS,
               quadrupole_linear=QUADRUPOLE_LINEAR) -> NativeParams:
        return NativeParams(float(beta), float(softening), float(cutoff), int(bool(quadrupole)), int(bool(periodic)),
                            float(box_length), float(prune_radius), float(quadrupole_radius),
                            float(quadrupole_linear))

    def force(self, *, beta: float = 2.0, softening: float = 1e-3, cutoff: float = 0.0, quadrupole: bool = True,
              periodic: bool = False, box_length: float = 1.0, prune_radius: float = 0.0,
              quadrupole_radius: float = QUADRUPOLE_RADIUS, quadrupole_linear: float = QUADRUPOLE_LINEAR,
              out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Softened self-gravity. periodic: minimum image in a cube of side
        box_length (monopole far field); cutoff > 0: the erfc short-range
        split; prune_radius > 0: skip cells beyond it (TreePM short range);
        quadrupole_radius: the quadrupole only within that many opening radii
        of the group (0: everywhere); quadrupole_linear: kappa of the
        once-per-group first-order quadrupole (0: exact everywhere)."""
        prm = self.params(beta, softening, cutoff, quadrupole, periodic, box_length, prune_radius, quadrupole_radius,
                          quadrupole_linear)
        out = out if out is not None else torch.empty((self.n, 3), dtype=torch.float32, device=self.device)
        _check(lib().sbh_native_force(_stream_ptr(self.device), ctypes.byref(prm), _p(out), _p(self.ws),
                                      self.ws.numel()), "native_force")
        return out

    def stochastic_force(self, *, beta: float = 2.0, beta_coarse: float = 1.0, samples: int = 32, seed: int = 0,
                         softening: float = 1e-3, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Stochastic Barnes-Hut self-gravity (Plummer softening): the group
        walk at beta_coarse plus, per target group, `samples` nodes of its
        coarse cut drawn in proportion to their octupole size and refined
        to beta (sbh_native_stochastic_force). Its expectation is
        force(beta=beta, quadrupole_radius=0, quadrupole_linear=0); the
        draws depend on the seed and each group's first input index."""
        prm = self.params(beta, softening, 0.0, True, False, 1.0, 0.0, 0.0, 0.0)
        out = out if out is not None else torch.empty((self.n, 3), dtype=torch.float32, device=self.device)
        _check(lib().sbh_native_stochastic_force(_stream_ptr(self.device), ctypes.byref(prm), float(beta_coarse),
                                                 int(samples), ctypes.c_uint64(int(seed) & (2 ** 64 - 1)), _p(out),
                                                 _p(self.ws), self.ws.numel()), "native_stochastic_force")
        return out

    def stochastic_force_vjp(self, cotangent, *, beta: float = 2.0, beta_coarse: float = 1.0, samples: int = 32,
                             seed: int = 0, softening: float = 1e-3, want_force: bool = True):
        """(estimate or None, d/d points, d/d masses) of sum(cotangent *
        stochastic_force(...)) at the same seed, the draws held fixed
        (sbh_native_stochastic_force_vjp; the tree built with_adjoint)."""
        prm = self.params(beta, softening, 0.0, True, False, 1.0, 0.0, 0.0, 0.0)
        cot = _f32(cotangent, self.device)
        if cot.shape != (self.n, 3):
            raise ValueError("cotangent must have shape (N, 3)")
        f = torch.empty((self.n, 3), dtype=torch.float32, device=self.device) if want_force else None
        gx = torch.empty((self.n, 3), dtype=torch.float32, device=self.device)
        gm = torch.empty(self.n, dtype=torch.float32, device=self.device)
        _check(lib().sbh_native_stochastic_force_vjp(_stream_ptr(self.device), ctypes.byref(prm), float(beta_coarse),
                                                     int(samples), ctypes.c_uint64(int(seed) & (2 ** 64 - 1)),
                                                     _p(cot), _p(f), _p(gx), _p(gm), _p(self.ws), self.ws.numel()),
               "native_stochastic_force_vjp")
        return f, gx, gm

    def force_vjp(self, cotangent, *, beta: float = 2.0, softening: float = 1e-3, cutoff: float = 0.0,
                  quadrupole: bool = True, periodic: bool = False, box_length: float = 1.0,
                  prune_radius: float = 0.0, quadrupole_radius: float = QUADRUPOLE_RADIUS,
                  quadrupole_linear: float = QUADRUPOLE_LINEAR, want_force: bool = True):
        """(force or None, d/d points, d/d masses) of sum(cotangent * force)."""
        prm = self.params(beta, softening, cutoff, quadrupole, periodic, box_length, prune_radius, quadrupole_radius,
                          quadrupole_linear)
        cot = _f32(cotangent, self.device)
        if cot.shape != (self.n, 3):
            raise ValueError("cotangent must have shape (N, 3)")
        f = torch.empty((self.n, 3), dtype=torch.float32, device=self.device) if want_force else None
        gx = torch.empty((self.n, 3), dtype=torch.float32, device=self.device)
        gm = torch.empty(self.n, dtype=torch.float32, device=self.device)
        _check(lib().sbh_native_force_vjp(_stream_ptr(self.device), ctypes.byref(prm), _p(cot), _p(f), _p(gx),
                                          _p(gm), _p(self.ws), self.ws.numel()), "native_force_vjp")
        return f, gx, gm

    def adjoint_walk(self, cotangent, params: NativeParams, force_out=None):
        """Phase 1 of force_vjp (the traversal)."""
        _check(lib().sbh_native_adjoint_walk(_stream_ptr(self.device), ctypes.byref(params), _p(cotangent),
                                             _p(force_out), _p(self.ws), self.ws.numel()), "native_adjoint_walk")

    def adjoint_finalize(self, grad_points, grad_masses):
        """Phase 2 of force_vjp (node adjoints to particles, input order)."""
        _check(lib().sbh_native_adjoint_finalize(_stream_ptr(self.device), _p(grad_points), _p(grad_masses),
                                                 _p(self.ws), self.ws.numel()), "native_adjoint_finalize")

    def query_side_gradient(self) -> torch.Tensor:
        """The query-side part J_i^T w_i of the last adjoint walk's gradient
        (n x 3, input order): the reference octree8 VJP's convention."""
        out = torch.empty((self.n, 3), dtype=torch.float32, device=self.device)
        _check(lib().sbh_native_adjoint_query_side(_stream_ptr(self.device), _p(out), _p(self.ws), self.ws.numel()),
               "native_adjoint_query_side")
        return out

    def winding_number(self, queries, *, beta: float = 2.0) -> torch.Tensor:
        q = _f32(queries, self.device)
        if q.ndim != 2 or q.shape[1] != 3:
            raise ValueError("queries must be (M, 3)")
        need = int(lib().sbh_native_query_workspace_bytes(q.shape[0]))
        if self.qws is None or self.qws.numel() < need:
            self.qws = torch.empty(max(need, 256), dtype=torch.uint8, device=self.device)
        out = torch.empty(q.shape[0], dtype=torch.float32, device=self.device)
        _check(lib().sbh_native_winding_number(_stream_ptr(self.device), float(beta), _p(q), q.shape[0], _p(out),
                                               _p(self.ws), self.ws.numel(), _p(self.qws), self.qws.numel()),
               "native_winding_number")
        return out

    def winding_number_vjp(self, queries, cotangent, *, beta: float = 2.0, want_value: bool = False):
        """(w or None, dL/dqueries (M, 3), dL/dpoints (N, 3), dL/dnormals
        (N, 3), dL/dmasses (N,)) of L = sum_i u_i w(q_i) for the cotangent u
        (M,); the tree must be built with normals and with_adjoint."""
        q = _f32(queries, self.device)
        u = _f32(cotangent, self.device)
        if q.ndim != 2 or q.shape[1] != 3:
            raise ValueError("queries must be (M, 3)")
        if u.shape != (q.shape[0],):
            raise ValueError("cotangent must have shape (M,)")
        need = int(lib().sbh_native_query_workspace_bytes(q.shape[0]))
        if self.qws is None or self.qws.numel() < need:
            self.qws = torch.empty(max(need, 256), dtype=torch.uint8, device=self.device)
        w = torch.empty(q.shape[0], dtype=torch.float32, device=self.device) if want_value else None
        gq = torch.empty((q.shape[0], 3), dtype=torch.float32, device=self.device)
        gp = torch.empty((self.n, 3), dtype=torch.float32, device=self.device)
        gn = torch.empty((self.n, 3), dtype=torch.float32, device=self.device)
        gm = torch.empty(self.n, dtype=torch.float32, device=self.device)
        _check(lib().sbh_native_winding_number_vjp(_stream_ptr(self.device), float(beta), _p(q), q.shape[0], _p(u),
                                                   _p(w), _p(gq), _p(gp), _p(gn), _p(gm), _p(self.ws),
                                                   self.ws.numel(), _p(self.qws), self.qws.numel()),
               "native_winding_number_vjp")
        return w, gq, gp, gn, gm

    def stats(self) -> dict:
        out = (ctypes.c_uint64 * 4)()
        rc = lib().sbh_native_stats(_stream_ptr(self.device), _p(self.ws), self.ws.numel(), out)
        _check(rc, "native_stats")
        fq = ctypes.c_uint64(0)
        _check(lib().sbh_native_quadrupole_count(_stream_ptr(self.device), _p(self.ws), self.ws.numel(),
                                                  ctypes.byref(fq)), "native_quadrupole_count")
        fc = (ctypes.c_uint64 * 3)()
        _check(lib().sbh_native_far_counts(_stream_ptr(self.device), _p(self.ws), self.ws.numel(), fc),
               "native_far_counts")
        return dict(nodes=int(out[0]), groups=int(out[1]), far=int(out[2]), near=int(out[3]),
                    far_quadrupole=int(fq.value), far_quadrupole_exact=int(fc[0]),
                    far_quadrupole_linear=int(fc[1]), linear_pairs=int(fc[2]))

    def export(self):
        """(sorted keys u64, permutation, node records (nn x 80 bytes)) as CPU numpy arrays."""
        nn = ctypes.c_uint64(0)
        _check(lib().sbh_native_export(_stream_ptr(self.device), _p(self.ws), self.ws.numel(), None, None, None, 0,
                                       ctypes.byref(nn)), "native_export")
        keys = torch.empty(self.n, dtype=torch.int64, device=self.device)
        perm = torch.empty(self.n, dtype=torch.int32, device=self.device)
        nodes = torch.empty(int(nn.value) * self.NODE_BYTES, dtype=torch.uint8, device=self.device)
        _check(lib().sbh_native_export(_stream_ptr(self.device), _p(self.ws), self.ws.numel(), _p(keys), _p(perm),
                                       _p(nodes), int(nn.value), ctypes.byref(nn)), "native_export")
        return (keys.cpu().numpy().view(np.uint64), perm.cpu().numpy().view(np.uint32),
                nodes.cpu().numpy().reshape(-1, self.NODE_BYTES))


def native_force(points, masses, *, beta: float = 2.0, softening: float = 1e-3, cutoff: float = 0.0,
                 leaf_size: int = 16, quadrupole: bool = True) -> torch.Tensor:
    """Softened self-gravity on the native tree (build + force)."""
    t = NativeTree().build(points, masses, leaf_size=leaf_size, with_adjoint=False)
    return t.force(beta=beta, softening=softening, cutoff=cutoff, quadrupole=quadrupole)


class _NativeGravity(torch.autograd.Function):
    """Self-gravity with the full adjoint. forward builds the tree and sums;
    backward rebuilds it from the saved inputs (recompute, like the
    reference's custom_vjp) and runs the adjoint walk: gradients w.r.t. both
    positions and masses."""

    @staticmethod
    def forward(ctx, points, masses, cfg):
        beta, soft, cut, leaf, quad = cfg
        ctx.save_for_backward(points, masses)
        ctx.cfg = cfg
        t = NativeTree().build(points.detach(), masses.detach(), leaf_size=leaf, with_adjoint=False)
        return t.force(beta=beta, softening=soft, cutoff=cut, quadrupole=quad)

    @staticmethod
    def backward(ctx, cot):
        points, masses = ctx.saved_tensors
        beta, soft, cut, leaf, quad = ctx.cfg
        t = NativeTree().build(points.detach(), masses.detach(), leaf_size=leaf, with_adjoint=True)
        _, gx, gm = t.force_vjp(cot.contiguous(), beta=beta, softening=soft, cutoff=cut, quadrupole=quad,
                                want_force=False)
        return gx, gm, None


# Candidate block sizes of autotune_octree8 (warps of 32 Morton-ordered
# queries per block in the warp-cooperative octree8 traversals).
AUTOTUNE_OCTREE8_THREADS = (64, 128, 256, 512)


def autotune_octree8(leaf_bytes, node_bytes, queries, *, candidates=AUTOTUNE_OCTREE8_THREADS, reps: int = 2,
                     **soft_kwargs) -> dict:
    """Picks the octree8 traversals' block size for this tree and these
    queries: times softened_barnes_hut_force_octree8 (soft_kwargs as its
    keywords) at each candidate `threads` and returns the fastest. The
    warp-cooperative traversal walks 32 Morton-ordered queries per warp with
    threads / 32 warps per block; its per-warp shared-memory stack holds 64
    entries for a dense octree8 of depth <= 9 and 128 otherwise. Results do
    not depend on the block size."""
    dev = _device()
    leaf, node, q = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _f32(queries, dev)
    trials = []
    for th in candidates:
        softened_barnes_hut_force_octree8(leaf, node, q, threads=int(th), **soft_kwargs)  # warm-up
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            softened_barnes_hut_force_octree8(leaf, node, q, threads=int(th), **soft_kwargs)
        b.record()
        torch.cuda.synchronize(dev)
        trials.append((a.elapsed_time(b) / reps, int(th)))
    ms, th = min(trials)
    return dict(threads=th, ms=ms, trials=[dict(threads=t_, ms=m_) for m_, t_ in trials])


# Candidate (leaf size, most targets per group) pairs of autotune_native:
# groups of 128 or 96 suit clustered systems, 64 near-uniform ones; leaves of
# 12 to 20 cost about the same on Plummer spheres.
AUTOTUNE_CANDIDATES = ((16, 128), (16, 96), (16, 64), (24, 64))


class _NativeWindingNumber(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, normals, masses, queries, cfg):
        beta, leaf = cfg
        t = NativeTree().build(points.detach(), masses.detach(), normals=normals.detach(), leaf_size=leaf,
                               with_adjoint=False)
        ctx.save_for_backward(points, normals, masses, queries)
        ctx.cfg = cfg
        return t.winding_number(queries.detach(), beta=beta)

    @staticmethod
    def backward(ctx, cot):
        points, normals, masses, queries = ctx.saved_tensors
        beta, leaf = ctx.cfg
        t = NativeTree().build(points.detach(), masses.detach(), normals=normals.detach(), leaf_size=leaf,
                               with_adjoint=True)
        _, gq, gp, gn, gm = t.winding_number_vjp(queries.detach(), cot.contiguous(), beta=beta)
        return gp, gn, gm, gq, None


def native_winding_number(points, normals, masses, queries, *, beta: float = 2.0, leaf_size: int = 16):
    """Generalized winding number of oriented points (points, normals,
    masses = area weights) at the queries, on the native tree; differentiable
    with respect to all four through the analytic adjoint walk (the tree is
    rebuilt in the backward pass, opening decisions recomputed)."""
    dev = _device()
    points, normals, masses, queries = (x if isinstance(x, torch.Tensor) else _f32(x, dev)
                                        for x in (points, normals, masses, queries))
    return _NativeWindingNumber.apply(points, normals, masses, queries, (float(beta), int(leaf_size)))


def autotune_native(points, masses, system_offsets=None, *, normals=None, adjoint: bool = True,
                    candidates=AUTOTUNE_CANDIDATES, reps: int = 2, **walk_kw) -> dict:
    """Times build + walk (force_vjp when adjoint, else force) of the given
    system(s) for each (leaf_size, group_size) candidate and returns the
    fastest as dict(leaf_size, group_size, ms, trials). Results do not
    depend on the choice beyond FP32 rounding and the opening decisions a
    group size implies; the walk parameters (beta, softening, ...) are the
    caller's."""
    dev = points.device if isinstance(points, torch.Tensor) and points.is_cuda else _device()
    tree = NativeTree(dev)
    cot = None
    trials = []
    for leaf, group in candidates:
        def step():
            tree.build(points, masses, normals, system_offsets, leaf_size=leaf, with_adjoint=adjoint,
                       group_size=group)
            if adjoint:
                return tree.force_vjp(cot, **walk_kw)
            return tree.force(**walk_kw)

        if cot is None:
            cot = torch.ones((int(points.shape[0]), 3), dtype=torch.float32, device=dev)
        step()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            step()
        b.record()
        torch.cuda.synchronize(dev)
        trials.append((a.elapsed_time(b) / reps, leaf, group))
    ms, leaf, group = min(trials)
    return dict(leaf_size=leaf, group_size=group, ms=ms,
                trials=[dict(leaf_size=l_, group_size=g_, ms=m_) for m_, l_, g_ in trials])


def native_force_recompute_vjp(points, masses, *, beta: float = 2.0, softening: float = 1e-3, cutoff: float = 0.0,
                               leaf_size: int = 16, quadrupole: bool = True) -> torch.Tensor:
    """Differentiable native self-gravity (gradients w.r.t. points and masses)."""
    if beta <= 0:
        raise ValueError("beta must be > 0")
    if softening < 0:
        raise ValueError("softening must be >= 0")
    dev = _device()
    points = points if isinstance(points, torch.Tensor) else _f32(points, dev)
    masses = masses if isinstance(masses, torch.Tensor) else _f32(masses, dev)
    return _NativeGravity.apply(points, masses, (float(beta), float(softening), float(cutoff), int(leaf_size),
                                                 bool(quadrupole)))


class _NativeStochasticGravity(torch.autograd.Function):
    """The native stochastic estimator with its adjoint: forward builds the
    tree and draws (seeded); backward rebuilds the tree from the saved inputs
    and runs the adjoint of the same draws (held fixed)."""

    @staticmethod
    def forward(ctx, points, masses, cfg):
        beta, beta_c, samples, seed, soft, leaf = cfg
        ctx.save_for_backward(points, masses)
        ctx.cfg = cfg
        t = NativeTree().build(points.detach(), masses.detach(), leaf_size=leaf, with_adjoint=False)
        return t.stochastic_force(beta=beta, beta_coarse=beta_c, samples=samples, seed=seed, softening=soft)

    @staticmethod
    def backward(ctx, cot):
        points, masses = ctx.saved_tensors
        beta, beta_c, samples, seed, soft, leaf = ctx.cfg
        t = NativeTree().build(points.detach(), masses.detach(), leaf_size=leaf, with_adjoint=True)
        _, gx, gm = t.stochastic_force_vjp(cot.contiguous(), beta=beta, beta_coarse=beta_c, samples=samples,
                                           seed=seed, softening=soft, want_force=False)
        return gx, gm, None


def native_stochastic_force(points, masses, *, beta: float = 2.0, beta_coarse: float = 1.0, samples: int = 32,
                            seed: int = 0, softening: float = 1e-3, leaf_size: int = 16) -> torch.Tensor:
    """Differentiable stochastic Barnes-Hut self-gravity on the native tree
    (NativeTree.stochastic_force; gradients w.r.t. points and masses with
    the draws of `seed` held fixed)."""
    if not 0 < beta_coarse <= beta:
        raise ValueError("beta_coarse must be in (0, beta]")
    if softening < 0:
        raise ValueError("softening must be >= 0")
    dev = _device()
    points = points if isinstance(points, torch.Tensor) else _f32(points, dev)
    masses = masses if isinstance(masses, torch.Tensor) else _f32(masses, dev)
    return _NativeStochasticGravity.apply(points, masses, (float(beta), float(beta_coarse), int(samples), int(seed),
                                                           float(softening), int(leaf_size)))


# ---------------------------------------------------------------------------
# level-3 tree and Node2 / Node3 targets (python/jax_sbh_ffi.py:744-862,
# 963-1334)
# ---------------------------------------------------------------------------
TREE_POTENTIAL, TREE_FORCE, TREE_SOFT_FORCE, TREE_WINDING = 0, 1, 2, 3
TREE_SMOOTHDIST = 6


def build_octree_buffers_with_contrib(points, normals, masses, min_corner=None, max_corner=None, *,
                                      alpha: float = 1.0, level: int = 3, backend: str = "ffi"):
    """Tree3DNode<1,3> buffers (python/jax_sbh_ffi.py:805-878).
    backend="ffi": root + up to 512 leaf children on the 8^3 grid of
    [min, max] (src/sbh_ffi.cu:736-1037). backend="cpu": the full adaptive
    tree of the reference's CPU builder sbh.Octree3 (leaf size 1, alpha 1,
    as the reference passes it), built here on the GPU with the same bytes."""
    del alpha
    if level != 3:
        raise ValueError("level must be 3 (FFI expects Tree3DNode<1, 3>)")
    if backend == "cpu":
        return _adaptive_tree(3, points, normals, masses, min_corner, max_corner, 1.0)
    if backend != "ffi":
        raise ValueError("backend must be 'ffi' or 'cpu'")
    dev = _device()
    points, normals, masses = _f32(points, dev), _f32(normals, dev), _f32(masses, dev)
    if points.ndim != 2 or points.shape[1] != 3:
        raise ValueError("points must have shape (N, 3)")
    if normals.shape != points.shape:
        raise ValueError("normals shape mismatch")
    if masses.ndim != 1 or masses.shape[0] != points.shape[0]:
        raise ValueError("masses must have shape (N,)")
    if points.shape[0] == 0 and (min_corner is None or max_corner is None):
        raise ValueError("empty point set needs explicit min_corner/max_corner")
    mn, mx = _default_corners(points, min_corner, max_corner, dev)
    n = points.shape[0]
    nmax = octree_level3_max_nodes()
    leaf = torch.empty(n * leaf3_size(), dtype=torch.uint8, device=dev)
    node = torch.empty(nmax * node3_size(), dtype=torch.uint8, device=dev)
    contrib = torch.empty(nmax * leaf3_size(), dtype=torch.uint8, device=dev)
    ws = workspace(int(lib().sbh_build_octree_level3_workspace_bytes(n)), dev)
    _check(lib().sbh_build_octree_level3(_stream_ptr(dev), _p(points), _p(normals), _p(masses), n, _p(mn), _p(mx),
                                         _p(leaf), leaf.numel(), _p(node), node.numel(), _p(contrib), contrib.numel(),
                                         _p(ws), ws.numel()), "build_octree_buffers")
    return leaf, node, contrib


def build_octree_buffers(points, normals, masses, min_corner=None, max_corner=None, *, alpha: float = 1.0,
                         level: int = 3, backend: str = "ffi"):
    leaf, node, _ = build_octree_buffers_with_contrib(points, normals, masses, min_corner, max_corner, alpha=alpha,
                                                      level=level, backend=backend)
    return leaf, node


NODE2_BYTES = 616
LEAF2_BYTES = 24


def _adaptive_tree(dim, points, normals, masses, min_corner, max_corner, alpha):
    """Leaf / node / contrib buffers of the reference's adaptive trees
    (Tree2D<1,3> for dim 2, Tree3D<1,3> for dim 3), built on the GPU."""
    dev = _device()
    points, masses = _f32(points, dev), _f32(masses, dev)
    if points.ndim != 2 or points.shape[1] != dim:
        raise ValueError(f"points must have shape (N, {dim})")
    normals = _f32(normals, dev) if normals is not None else torch.zeros_like(points)
    if normals.shape != points.shape:
        raise ValueError("normals shape mismatch")
    if masses.ndim != 1 or masses.shape[0] != points.shape[0]:
        raise ValueError("masses must have shape (N,)")
    n = points.shape[0]
    if n == 0:
        raise ValueError("the tree needs at least one point")
    mn, mx = _default_corners(points, min_corner, max_corner, dev)
    node_b, leaf_b = (NODE2_BYTES, LEAF2_BYTES) if dim == 2 else (node3_size(), leaf3_size())
    build = lib().sbh_build_quadtree if dim == 2 else lib().sbh_build_adaptive_octree
    wsb = lib().sbh_build_quadtree_workspace_bytes if dim == 2 else lib().sbh_build_adaptive_octree_workspace_bytes
    leaf = torch.empty(n * leaf_b, dtype=torch.uint8, device=dev)
    ws = workspace(int(wsb(n)), dev)
    cap = n + n // 2 + 64
    while True:
        node = torch.empty(cap * node_b, dtype=torch.uint8, device=dev)
        contrib = torch.empty(cap * leaf_b, dtype=torch.uint8, device=dev)
        nn = ctypes.c_uint64(0)
        rc = build(_stream_ptr(dev), _p(points), _p(normals), _p(masses), n, _p(mn), _p(mx), float(alpha), _p(leaf),
                   leaf.numel(), _p(node), node.numel(), _p(contrib), contrib.numel(), ctypes.byref(nn), _p(ws),
                   ws.numel())
        if rc == SBH_ERR_LIMIT and nn.value > cap:
            cap = int(nn.value)
            continue
        _check(rc, "build_quadtree_buffers" if dim == 2 else "build_octree_buffers")
        k = int(nn.value)
        return leaf, node[:k * node_b], contrib[:k * leaf_b]


def build_quadtree_buffers_with_contrib(points, normals, masses, min_corner=None, max_corner=None, *,
                                       alpha: float = 1.0, level: int = 3):
    """The adaptive quadtree Tree2DNode<1,3> (leaf size 1, 8 x 8 split per
    node) as (leaf_bytes, node_bytes, contrib_bytes) uint8 device tensors,
    built on the GPU with the bytes of the reference's CPU builder
    sbh.Quadtree3 (python/jax_sbh_ffi.py:692-742, include/tree2d.h)."""
    if level != 3:
        raise ValueError("level must be 3 (FFI expects Tree2DNode<1, 3>)")
    return _adaptive_tree(2, points, normals, masses, min_corner, max_corner, alpha)


def build_quadtree_buffers(points, normals, masses, min_corner=None, max_corner=None, *, alpha: float = 1.0,
                           level: int = 3):
    leaf, node, _ = build_quadtree_buffers_with_contrib(points, normals, masses, min_corner, max_corner, alpha=alpha,
                                                        level=level)
    return leaf, node


def _tree_call(kernel, leaf_bytes, node_bytes, queries, beta, softening_scale, cutoff_scale, periodic, box_length,
               threads, check_status=False):
    dev = _device()
    leaf, node, queries = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _f32(queries, dev)
    if queries.ndim != 2 or queries.shape[1] not in (2, 3):
        raise ValueError("queries must be (M, 2) or (M, 3)")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")
    dim = queries.shape[1]
    vec = kernel in (TREE_FORCE, TREE_SOFT_FORCE)
    out = torch.empty((queries.shape[0], dim) if vec else queries.shape[0], dtype=torch.float32, device=dev)
    ws = workspace(int(lib().sbh_traversal_workspace_bytes()), dev)
    _check(lib().sbh_barnes_hut_tree(_stream_ptr(dev), dim, kernel, _p(leaf), leaf.numel(), _p(node), node.numel(),
                                     _p(queries), queries.shape[0], _p(out), float(beta), float(softening_scale),
                                     float(cutoff_scale), int(bool(periodic)), float(box_length), int(threads), _p(ws),
                                     ws.numel()), "barnes_hut_tree")
    _status_after(ws, "barnes_hut_tree", check_status)
    return out


def barnes_hut_gravity(leaf_bytes, node_bytes, queries, *, beta: float = 2.0, periodic: bool = False,
                       box_length: float = 1.0, threads: int = 64):
    return _tree_call(TREE_POTENTIAL, leaf_bytes, node_bytes, queries, beta, 0.0, 1.0, periodic, box_length, threads)


def barnes_hut_force(leaf_bytes, node_bytes, queries, *, beta: float = 2.0, periodic: bool = False,
                     box_length: float = 1.0, threads: int = 256):
    return _tree_call(TREE_FORCE, leaf_bytes, node_bytes, queries, beta, 0.0, 1.0, periodic, box_length, threads)


def softened_barnes_hut_force(leaf_bytes, node_bytes, queries, *, beta: float = 2.0, softening_scale: float = 1e-2,
                              cutoff_scale: float = 1.0, periodic: bool = False, box_length: float = 1.0,
                              threads: int = 256):
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    return _tree_call(TREE_SOFT_FORCE, leaf_bytes, node_bytes, queries, beta, softening_scale, cutoff_scale, periodic,
                      box_length, threads)


def _tree_vjp_call(softened, leaf_bytes, node_bytes, queries, cotangent, beta, softening_scale, cutoff_scale, periodic,
                   box_length, threads):
    dev = _device()
    leaf, node, queries = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _f32(queries, dev)
    cot = _f32(cotangent, dev)
    if queries.ndim != 2 or queries.shape[1] not in (2, 3):
        raise ValueError("queries must be (M, 2) or (M, 3)")
    if cot.shape != queries.shape:
        raise ValueError("cotangent must have same shape as queries")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")
    out = torch.empty(queries.shape, dtype=torch.float32, device=dev)
    ws = workspace(int(lib().sbh_traversal_workspace_bytes()), dev)
    _check(lib().sbh_barnes_hut_tree_vjp(_stream_ptr(dev), queries.shape[1], int(softened), _p(leaf), leaf.numel(),
                                         _p(node), node.numel(), _p(queries), queries.shape[0], _p(cot), _p(out),
                                         float(beta), float(softening_scale), float(cutoff_scale), int(bool(periodic)),
                                         float(box_length), int(threads), _p(ws), ws.numel()), "barnes_hut_tree_vjp")
    return out


def barnes_hut_force_vjp(leaf_bytes, node_bytes, queries, cotangent, *, beta: float = 2.0, periodic: bool = False,
                         box_length: float = 1.0, threads: int = 256):
    """Analytic query-side VJP of barnes_hut_force with the forward's opening
    decisions (the reference's function of this name takes central finite
    differences, python/jax_sbh_ffi.py:1037-1060)."""
    return _tree_vjp_call(False, leaf_bytes, node_bytes, queries, cotangent, beta, 0.0, 1.0, periodic, box_length,
                          threads)


def softened_barnes_hut_force_vjp(leaf_bytes, node_bytes, queries, cotangent, *, beta: float = 2.0,
                                  softening_scale: float = 1e-2, cutoff_scale: float = 1.0, periodic: bool = False,
                                  box_length: float = 1.0, threads: int = 256):
    """Analytic query-side VJP of softened_barnes_hut_force (finite
    differences in the reference, python/jax_sbh_ffi.py:1108-1135)."""
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    return _tree_vjp_call(True, leaf_bytes, node_bytes, queries, cotangent, beta, softening_scale, cutoff_scale,
                          periodic, box_length, threads)


def barnes_hut_winding_number(leaf_bytes, node_bytes, queries, *, beta: float = 2.0, threads: int = 256):
    """Winding number on a Node2/Node3 tree (new target; the reference has it
    only in its pybind module, src/sbh_gpu.cu:100-120)."""
    return _tree_call(TREE_WINDING, leaf_bytes, node_bytes, queries, beta, 0.0, 1.0, False, 1.0, threads)


def _stochastic_tree_call(kernel, leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain, seed,
                          softening_scale, cutoff_scale, periodic, box_length, threads):
    dev = _device()
    leaf, node, contrib = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _u8(contrib_bytes, dev)
    queries = _f32(queries, dev)
    if queries.ndim != 2 or queries.shape[1] not in (2, 3):
        raise ValueError("queries must be (M, 2) or (M, 3)")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")
    if samples_per_subdomain < 1:
        raise ValueError("samples_per_subdomain must be >= 1")
    dim = queries.shape[1]
    vec = kernel in (TREE_FORCE, TREE_SOFT_FORCE)
    out = torch.empty((queries.shape[0], dim) if vec else queries.shape[0], dtype=torch.float32, device=dev)
    ws = workspace(int(lib().sbh_traversal_workspace_bytes()), dev)
    _check(lib().sbh_stochastic_bh_tree(_stream_ptr(dev), dim, kernel, _p(leaf), leaf.numel(), _p(node), node.numel(),
                                        _p(contrib), contrib.numel(), _p(queries), queries.shape[0], _p(out),
                                        int(samples_per_subdomain), int(seed), float(softening_scale),
                                        float(cutoff_scale), int(bool(periodic)), float(box_length), int(threads),
                                        _p(ws), ws.numel()), "stochastic_bh_tree")
    return out


def stochastic_barnes_hut_gravity(leaf_bytes, node_bytes, contrib_bytes, queries, *, samples_per_subdomain: int = 1,
                                  seed: int = 0, periodic: bool = False, box_length: float = 1.0, threads: int = 256):
    return _stochastic_tree_call(TREE_POTENTIAL, leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain,
                                 seed, 0.0, 1.0, periodic, box_length, threads)


def stochastic_barnes_hut_force(leaf_bytes, node_bytes, contrib_bytes, queries, *, samples_per_subdomain: int = 1,
                                seed: int = 0, periodic: bool = False, box_length: float = 1.0, threads: int = 256):
    return _stochastic_tree_call(TREE_FORCE, leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain,
                                 seed, 0.0, 1.0, periodic, box_length, threads)


def softened_stochastic_barnes_hut_force(leaf_bytes, node_bytes, contrib_bytes, queries, *,
                                         samples_per_subdomain: int = 1, seed: int = 0, softening_scale: float = 1e-2,
                                         cutoff_scale: float = 1.0, periodic: bool = False, box_length: float = 1.0,
                                         threads: int = 256):
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    return _stochastic_tree_call(TREE_SOFT_FORCE, leaf_bytes, node_bytes, contrib_bytes, queries,
                                 samples_per_subdomain, seed, softening_scale, cutoff_scale, periodic, box_length,
                                 threads)


def _stochastic_tree_vjp_call(softened, leaf_bytes, node_bytes, contrib_bytes, queries, cotangent,
                              samples_per_subdomain, seed, softening_scale, cutoff_scale, periodic, box_length,
                              threads):
    dev = _device()
    leaf, node, contrib = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _u8(contrib_bytes, dev)
    queries, cot = _f32(queries, dev), _f32(cotangent, dev)
    if queries.ndim != 2 or queries.shape[1] not in (2, 3):
        raise ValueError("queries must be (M, 2) or (M, 3)")
    if cot.shape != queries.shape:
        raise ValueError("cotangent must have same shape as queries")
    if periodic and box_length <= 0:
        raise ValueError("box_length must be > 0 when periodic=True")
    if threads < 1:
        raise ValueError("threads must be >= 1")
    if samples_per_subdomain < 1:
        raise ValueError("samples_per_subdomain must be >= 1")
    out = torch.empty(queries.shape, dtype=torch.float32, device=dev)
    ws = workspace(int(lib().sbh_traversal_workspace_bytes()), dev)
    _check(lib().sbh_stochastic_bh_tree_vjp(_stream_ptr(dev), queries.shape[1], int(softened), _p(leaf), leaf.numel(),
                                            _p(node), node.numel(), _p(contrib), contrib.numel(), _p(queries),
                                            queries.shape[0], _p(cot), _p(out), int(samples_per_subdomain), int(seed),
                                            float(softening_scale), float(cutoff_scale), int(bool(periodic)),
                                            float(box_length), int(threads), _p(ws), ws.numel()),
           "stochastic_bh_tree_vjp")
    return out


def stochastic_barnes_hut_force_vjp(leaf_bytes, node_bytes, contrib_bytes, queries, cotangent, *,
                                    samples_per_subdomain: int = 1, seed: int = 0, periodic: bool = False,
                                    box_length: float = 1.0, threads: int = 256):
    """Query-side VJP of stochastic_barnes_hut_force with the forward's
    sampled paths and weights for the same seed (finite differences in the
    reference, python/jax_sbh_ffi.py:1222-1250)."""
    return _stochastic_tree_vjp_call(False, leaf_bytes, node_bytes, contrib_bytes, queries, cotangent,
                                     samples_per_subdomain, seed, 0.0, 1.0, periodic, box_length, threads)


def softened_stochastic_barnes_hut_force_vjp(leaf_bytes, node_bytes, contrib_bytes, queries, cotangent, *,
                                             samples_per_subdomain: int = 1, seed: int = 0,
                                             softening_scale: float = 1e-2, cutoff_scale: float = 1.0,
                                             periodic: bool = False, box_length: float = 1.0, threads: int = 256):
    """Query-side VJP of softened_stochastic_barnes_hut_force (finite
    differences in the reference, python/jax_sbh_ffi.py:1302-1334)."""
    _check_soft(softening_scale, cutoff_scale, periodic, box_length, threads)
    return _stochastic_tree_vjp_call(True, leaf_bytes, node_bytes, contrib_bytes, queries, cotangent,
                                     samples_per_subdomain, seed, softening_scale, cutoff_scale, periodic, box_length,
                                     threads)


def stochastic_barnes_hut_winding_number(leaf_bytes, node_bytes, contrib_bytes, queries, *,
                                         samples_per_subdomain: int = 1, seed: int = 0, threads: int = 256):
    return _stochastic_tree_call(TREE_WINDING, leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain,
                                 seed, 0.0, 1.0, False, 1.0, threads)


# ---------------------------------------------------------------------------
# the reference's pybind module sbh_gpu (src/sbh_gpu.cu:566-661): scalar
# kernels on Node2/Node3 trees by brute force, warp-vote BH and MLPCV. The
# module wraps a CPU-built tree object; here the tree is its buffers (from
# build_quadtree_buffers_with_contrib or build_octree_buffers_with_contrib).
# Each returns (values, milliseconds on the GPU), as the module does.
# ---------------------------------------------------------------------------
def _timed(fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    e1.synchronize()
    return out, e0.elapsed_time(e1)


def _brute(kind, leaf_bytes, queries):
    dev = _device()
    leaf, queries = _u8(leaf_bytes, dev), _f32(queries, dev)
    if queries.ndim != 2 or queries.shape[1] not in (2, 3):
        raise ValueError("queries must be (M, 2) or (M, 3)")
    out = torch.empty(queries.shape[0], dtype=torch.float32, device=dev)

    def run():
        _check(lib().sbh_brute_force_tree(_stream_ptr(dev), queries.shape[1], kind, _p(leaf), leaf.numel(),
                                          _p(queries), queries.shape[0], _p(out), 32), "brute_force_tree")
        return out
    return _timed(run)


def eval_brute_force_gravity(leaf_bytes, queries):
    return _brute(TREE_POTENTIAL, leaf_bytes, queries)


def eval_brute_force_wn(leaf_bytes, queries):
    return _brute(TREE_WINDING, leaf_bytes, queries)


def eval_brute_force_smoothdist(leaf_bytes, queries):
    return _brute(TREE_SMOOTHDIST, leaf_bytes, queries)


def eval_barnes_hut_gravity(leaf_bytes, node_bytes, queries, beta: float):
    return _timed(lambda: _tree_call(TREE_POTENTIAL, leaf_bytes, node_bytes, queries, beta, 0.0, 1.0, False, 1.0, 32))


def eval_barnes_hut_wn(leaf_bytes, node_bytes, queries, beta: float):
    return _timed(lambda: _tree_call(TREE_WINDING, leaf_bytes, node_bytes, queries, beta, 0.0, 1.0, False, 1.0, 32))


def eval_barnes_hut_smoothdist(leaf_bytes, node_bytes, queries, beta: float):
    return _timed(lambda: _tree_call(TREE_SMOOTHDIST, leaf_bytes, node_bytes, queries, beta, 0.0, 1.0, False, 1.0,
                                     32))


def _mlpcv_shared_seed(kind, leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain):
    dev = _device()
    leaf, node, contrib = _u8(leaf_bytes, dev), _u8(node_bytes, dev), _u8(contrib_bytes, dev)
    queries = _f32(queries, dev)
    if queries.ndim != 2 or queries.shape[1] not in (2, 3):
        raise ValueError("queries must be (M, 2) or (M, 3)")
    out = torch.empty(queries.shape[0], dtype=torch.float32, device=dev)
    ws = workspace(int(lib().sbh_traversal_workspace_bytes()), dev)

    def run():
        _check(lib().sbh_stochastic_bh_tree_shared_seed(_stream_ptr(dev), queries.shape[1], kind, _p(leaf),
                                                        leaf.numel(), _p(node), node.numel(), _p(contrib),
                                                        contrib.numel(), _p(queries), queries.shape[0], _p(out),
                                                        int(samples_per_subdomain), 0, 32, _p(ws), ws.numel()),
               "stochastic_bh_tree_shared_seed")
        return out
    return _timed(run)


def multi_level_prefix_control_variate_gravity(leaf_bytes, node_bytes, contrib_bytes, queries,
                                               samples_per_subdomain: int):
    return _mlpcv_shared_seed(TREE_POTENTIAL, leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain)


def multi_level_prefix_control_variate_wn(leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain: int):
    return _mlpcv_shared_seed(TREE_WINDING, leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain)


def multi_level_prefix_control_variate_smoothdist(leaf_bytes, node_bytes, contrib_bytes, queries,
                                                  samples_per_subdomain: int):
    return _mlpcv_shared_seed(TREE_SMOOTHDIST, leaf_bytes, node_bytes, contrib_bytes, queries, samples_per_subdomain)
