"""ctypes bindings for the oracle -- TEST INFRASTRUCTURE ONLY.

Loads the project's C restatement (``_ref/libsbh_oracle.so``, built from
``sbh_oracle.c``) and, when present, the reference's own code compiled by
``Makefile``'s ``ref`` target:

* ``_ref/libsbh_ref_cpu.so`` / ``libsbh_ref_cpu64.so``: the reference's CPU
  ``Tree3D``/``Tree2D`` build and ``evaluateBarnesHut_stackless`` driven like
  ``src/sbh.cpp:49-88`` (FP32 and ``-DUSE_DOUBLE`` builds);
* ``_ref/libsbh_ref_gpu.so``: the reference's ``src/sbh_ffi.cu`` handlers,
  callable with device pointers (GPU box only).

Only tests, the smoke check and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF = os.path.join(_HERE, "_ref")

_c_f = ctypes.c_float
_c_d = ctypes.c_double
_c_i = ctypes.c_int
_c_i64 = ctypes.c_int64
_c_p = ctypes.c_void_p
_c_u32 = ctypes.c_uint32
_c_sz = ctypes.c_size_t

_LIBS: dict = {}


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(_c_p)


def lib_path(name: str) -> str:
    return os.path.join(_REF, name)


def available(name: str) -> bool:
    return os.path.exists(lib_path(name))


def _load(name: str) -> ctypes.CDLL:
    if name not in _LIBS:
        path = lib_path(name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library {path} is missing; run `make -C oracle` (and `make -C oracle ref`)")
        _LIBS[name] = ctypes.CDLL(path)
    return _LIBS[name]


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


# ---------------------------------------------------------------------------
# project restatement (libsbh_oracle.so)
# ---------------------------------------------------------------------------
def _orc() -> ctypes.CDLL:
    lib = _load("libsbh_oracle.so")
    if not getattr(lib, "_typed", False):
        lib.orc_octree8_total_nodes.restype = _c_u32
        lib.orc_octree8_total_nodes.argtypes = [_c_i]
        lib.orc_leaf3_size.restype = _c_sz
        lib.orc_octree8_node_size.restype = _c_sz
        lib.orc_direct_force_soft.argtypes = [_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_d, _c_d, _c_i, _c_d, _c_p]
        lib.orc_direct_force_soft_vjp.argtypes = [_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_d, _c_d, _c_i, _c_d, _c_p]
        lib.orc_direct_full_adjoint.argtypes = [_c_p, _c_p, _c_i64, _c_p, _c_d, _c_d, _c_p, _c_i64, _c_p, _c_p]
        lib.orc_bruteforce_gravity.argtypes = [_c_p, _c_p, _c_i64, _c_i, _c_p, _c_i64, _c_i, _c_d, _c_p]
        lib.orc_direct_winding_number.argtypes = [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p]
        lib.orc_build_octree8.restype = _c_i
        lib.orc_build_octree8.argtypes = [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_i, _c_p, _c_p, _c_p, _c_p, _c_p]
        lib.orc_bh_octree8.restype = _c_i
        lib.orc_bh_octree8.argtypes = [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_f, _c_i, _c_d, _c_d, _c_i, _c_f, _c_i, _c_f, _c_p, _c_p]
        lib.orc_native_sort.argtypes = [_c_p, _c_i64, _c_p, _c_p, _c_p]
        lib.orc_native_topology.restype = _c_i64
        lib.orc_native_topology.argtypes = [_c_p, _c_i64, _c_i, _c_p, _c_p, _c_p, _c_p]
        lib.orc_native_build.restype = _c_p
        lib.orc_native_build.argtypes = [_c_p, _c_i64, _c_i]
        lib.orc_native_free.argtypes = [_c_p]
        lib.orc_native_num_nodes.restype = _c_i64
        lib.orc_native_num_nodes.argtypes = [_c_p]
        lib.orc_native_get.argtypes = [_c_p] + [_c_p] * 9
        lib.orc_native_plan.restype = _c_i64
        lib.orc_native_plan.argtypes = [_c_p, _c_p, _c_p, _c_d, _c_i]
        lib.orc_native_eval.argtypes = [_c_p, _c_p, _c_p, _c_d, _c_d, _c_i, _c_p, _c_p, _c_p]
        lib.orc_native_set_periodic.argtypes = [_c_i, _c_f, _c_f]
        lib.orc_native_set_quadrupole_radius.argtypes = [_c_f]
        lib.orc_native_quadrupole_interactions.argtypes = [_c_p]
        lib.orc_native_quadrupole_interactions.restype = _c_i64
        lib.orc_native_adjoint.argtypes = [_c_p, _c_p, _c_p, _c_p, _c_d, _c_d, _c_i, _c_p, _c_p]
        lib.orc_native_plan_stats.argtypes = [_c_p, _c_p, _c_p, _c_p]
        lib.orc_native_fd.argtypes = [_c_p, _c_p, _c_p, _c_p, _c_d, _c_i, _c_p, _c_i64, _c_d, _c_d, _c_p, _c_p]
        lib.orc_native_set_quad_linear.argtypes = [_c_f]
        lib.orc_native_linear_quadrupole_counts.argtypes = [_c_p, _c_p, _c_p]
        lib.orc_native_wn_plan.restype = _c_i64
        lib.orc_native_wn_plan.argtypes = [_c_p, _c_p, _c_p, _c_p, _c_i64, _c_d]
        lib.orc_native_wn_eval.argtypes = [_c_p, _c_p, _c_p, _c_p, _c_p, _c_p]
        lib.orc_native_wn_adjoint.argtypes = [_c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p]
        lib.orc_native_records.argtypes = [_c_p, _c_p, _c_p, _c_p]
        lib.orc_native_stochastic_plan.restype = _c_i64
        lib.orc_native_stochastic_plan.argtypes = [_c_p, _c_p, _c_p, _c_i, _c_f, _c_f, _c_f, _c_i, ctypes.c_uint64]
        lib.orc_native_stochastic.restype = _c_i64
        lib.orc_native_stochastic.argtypes = [_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_i, _c_f, _c_f, _c_f, _c_i,
                                              ctypes.c_uint64, _c_p, _c_p]
        lib._typed = True
    return lib


def octree8_total_nodes(max_depth: int) -> int:
    return int(_orc().orc_octree8_total_nodes(int(max_depth)))


def direct_force_soft(points, masses, queries, eps, cutoff=0.0, periodic=False, box=1.0):
    """Softened direct force in double (src/sbh_ffi.cu:431-522); cutoff <= 0 is off."""
    p, m, q = _f32(points), _f32(masses), _f32(queries)
    out = np.zeros((q.shape[0], 3), np.float64)
    _orc().orc_direct_force_soft(_ptr(p), _ptr(m), p.shape[0], _ptr(q), q.shape[0], eps, cutoff,
                                 int(periodic), box, _ptr(out))
    return out


def direct_force_soft_vjp(points, masses, queries, cot, eps, cutoff=0.0, periodic=False, box=1.0):
    p, m, q, g = _f32(points), _f32(masses), _f32(queries), _f32(cot)
    out = np.zeros((q.shape[0], 3), np.float64)
    _orc().orc_direct_force_soft_vjp(_ptr(p), _ptr(m), p.shape[0], _ptr(q), q.shape[0], _ptr(g), eps,
                                     cutoff, int(periodic), box, _ptr(out))
    return out


def direct_full_adjoint(points, masses, w, eps, cutoff=0.0, idx=None):
    """Exact d/d(x, m) of sum_i w_i . a_i for self-gravity (double)."""
    p, m, ww = _f32(points), _f32(masses), _f32(w)
    if idx is None:
        nk = p.shape[0]
        ip = None
    else:
        ip = np.ascontiguousarray(np.asarray(idx, np.int64))
        nk = ip.shape[0]
    dx = np.zeros((nk, 3), np.float64)
    dm = np.zeros(nk, np.float64)
    _orc().orc_direct_full_adjoint(_ptr(p), _ptr(m), p.shape[0], _ptr(ww), eps, cutoff, _ptr(ip), nk,
                                   _ptr(dx), _ptr(dm))
    return dx, dm


def bruteforce_gravity(points, masses, queries, periodic=False, box=1.0):
    p, m, q = _f32(points), _f32(masses), _f32(queries)
    out = np.zeros(q.shape[0], np.float64)
    _orc().orc_bruteforce_gravity(_ptr(p), _ptr(m), p.shape[0], p.shape[1], _ptr(q), q.shape[0],
                                  int(periodic), box, _ptr(out))
    return out


def direct_winding_number(points, normals, masses, queries):
    p, nr, m, q = _f32(points), _f32(normals), _f32(masses), _f32(queries)
    out = np.zeros(q.shape[0], np.float64)
    _orc().orc_direct_winding_number(_ptr(p), _ptr(nr), _ptr(m), p.shape[0], _ptr(q), q.shape[0], _ptr(out))
    return out


def build_octree8(points, normals, masses, min_corner, max_corner, max_depth):
    """Reference-layout octree8 buffers (leaf, node, contrib bytes) + codes + perm."""
    p, nr, m = _f32(points), _f32(normals), _f32(masses)
    mn, mx = _f32(min_corner), _f32(max_corner)
    n = p.shape[0]
    total = octree8_total_nodes(max_depth)
    leaf = np.zeros(n * 32, np.uint8)
    node = np.zeros(total * 104, np.uint8)
    contrib = np.zeros(total * 32, np.uint8)
    codes = np.zeros(n, np.uint32)
    perm = np.zeros(n, np.int64)
    rc = _orc().orc_build_octree8(_ptr(p), _ptr(nr), _ptr(m), n, _ptr(mn), _ptr(mx), int(max_depth),
                                  _ptr(leaf), _ptr(node), _ptr(contrib), _ptr(codes), _ptr(perm))
    if rc != 0:
        raise ValueError("oracle octree8 build rejected its arguments")
    return leaf, node, contrib, codes, perm


KERNEL_GRAV_GRAD = 0
KERNEL_SOFT = 1
KERNEL_SOFT_VJP = 2


def bh_octree8(leaf, node, queries, beta, kernel, eps=0.0, cutoff=0.0, prune_enabled=False,
               prune_r_cut_mult=4.0, periodic=False, box=1.0, cot=None):
    """Classic BH on octree8 bytes (src/sbh_ffi.cu:1950-2144), double sums."""
    q = _f32(queries)
    leaf = np.ascontiguousarray(np.asarray(leaf, np.uint8))
    node = np.ascontiguousarray(np.asarray(node, np.uint8))
    g = _f32(cot) if cot is not None else None
    prune_on = 1 if (prune_enabled and cutoff > 0.0) else 0
    r_cut = np.float32(prune_r_cut_mult) * np.float32(cutoff) if prune_on else np.float32(0.0)
    r_cut_sq = float(np.float32(r_cut) * np.float32(r_cut))
    out = np.zeros((q.shape[0], 3), np.float64)
    counts = np.zeros(q.shape[0], np.int32)
    rc = _orc().orc_bh_octree8(_ptr(leaf), _ptr(node), _ptr(q), q.shape[0], _ptr(g), float(beta), int(kernel),
                               float(eps), float(cutoff), prune_on, r_cut_sq, int(periodic), float(box),
                               _ptr(out), _ptr(counts))
    if rc != 0:
        raise RuntimeError("oracle octree8 traversal overflowed its 128-entry stack")
    return out, counts


# ----------------------------- native tree -----------------------------------
def native_sort(points):
    p = _f32(points)
    n = p.shape[0]
    keys = np.zeros(n, np.uint64)
    perm = np.zeros(n, np.int64)
    box = np.zeros(4, np.float32)
    _orc().orc_native_sort(_ptr(p), n, _ptr(keys), _ptr(perm), _ptr(box))
    return keys, perm, box


class NativeTree:
    """The project's adaptive Morton octree, restated on the CPU."""

    def __init__(self, points, masses, leaf_size=16):
        self.points = _f32(points)
        self.masses = _f32(masses)
        self.leaf_size = int(leaf_size)
        self._lib = _orc()
        self._h = self._lib.orc_native_build(_ptr(self.points), self.points.shape[0], self.leaf_size)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.orc_native_free(self._h)
            self._h = None

    @property
    def num_nodes(self) -> int:
        return int(self._lib.orc_native_num_nodes(self._h))

    def arrays(self) -> dict:
        n, nn = self.points.shape[0], self.num_nodes
        a = dict(keys=np.zeros(n, np.uint64), perm=np.zeros(n, np.int64), start=np.zeros(nn, np.int32),
                 end=np.zeros(nn, np.int32), skip=np.zeros(nn, np.int32), level=np.zeros(nn, np.int8),
                 center=np.zeros((nn, 3), np.float32), side=np.zeros(nn, np.float32),
                 box=np.zeros(4, np.float32))
        self._lib.orc_native_get(self._h, *[_ptr(a[k]) for k in
                                            ("keys", "perm", "start", "end", "skip", "level", "center", "side", "box")])
        return a

    def plan(self, beta, group_size=32) -> int:
        """Record the traversal plan (beta = 1/theta); returns the interaction count."""
        return int(self._lib.orc_native_plan(self._h, _ptr(self.points), _ptr(self.masses), float(beta),
                                             int(group_size)))

    def quadrupole_interactions(self) -> int:
        """Far interactions (per target) of the plan that take the quadrupole."""
        return int(self._lib.orc_native_quadrupole_interactions(self._h))

    def linear_quadrupole_counts(self):
        """(far interactions per target with the linearized quadrupole, the
        (group, node) pairs they come from) of the recorded plan."""
        a, b = _c_i64(), _c_i64()
        self._lib.orc_native_linear_quadrupole_counts(self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def wn_plan(self, queries, beta) -> int:
        """Record the winding-number plan of external queries (the CUDA
        walk's query groups of 32); returns the interaction count."""
        self.queries = _f32(queries)
        return int(self._lib.orc_native_wn_plan(self._h, _ptr(self.points), _ptr(self.masses), _ptr(self.queries),
                                                self.queries.shape[0], float(beta)))

    def wn_eval(self, normals, points=None, masses=None, queries=None):
        """Winding number at the planned queries (float64), for possibly
        perturbed points, normals, masses and queries (plan frozen)."""
        p = self.points if points is None else _f32(points)
        m = self.masses if masses is None else _f32(masses)
        q = self.queries if queries is None else _f32(queries)
        out = np.zeros(q.shape[0], np.float64)
        self._lib.orc_native_wn_eval(self._h, _ptr(p), _ptr(_f32(normals)), _ptr(m), _ptr(q), _ptr(out))
        return out

    def wn_adjoint(self, normals, u):
        """(dq, dp, dn, dm) of sum_i u_i w(q_i) with the plan frozen (float64)."""
        nq, n = self.queries.shape[0], self.points.shape[0]
        dq, dp, dn = np.zeros((nq, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        dm = np.zeros(n)
        self._lib.orc_native_wn_adjoint(self._h, _ptr(self.points), _ptr(_f32(normals)), _ptr(self.masses),
                                        _ptr(self.queries), _ptr(_f32(u)), _ptr(dq), _ptr(dp), _ptr(dn), _ptr(dm))
        return dq, dp, dn, dm

    def node_records(self) -> np.ndarray:
        """Node records in the GPU's layout (nn x 80 bytes) from this tree."""
        out = np.zeros((self.num_nodes, 80), np.uint8)
        self._lib.orc_native_records(self._h, _ptr(self.points), _ptr(self.masses), _ptr(out))
        return out

    def stochastic_plan(self, node_records, *, group_size=128, beta_coarse=1.0, beta=2.0, softening=1e-3,
                        samples=32, seed=0) -> int:
        """Record the native stochastic estimator's terms at this seed as the
        plan (orc_native_stochastic_plan: coefficients per term, decisions
        and draws taken on node_records, the GPU export); force(quad=True),
        adjoint(quad=True) and finite_differences(quad=True) then evaluate
        the estimate and its VJP with the draws held fixed."""
        nodes = np.ascontiguousarray(np.asarray(node_records, np.uint8))
        eps2 = np.float32(np.float32(softening) * np.float32(softening) + np.float32(1e-12))
        return int(self._lib.orc_native_stochastic_plan(self._h, _ptr(self.points), _ptr(nodes), int(group_size),
                                                        float(beta_coarse), float(beta), float(eps2), int(samples),
                                                        ctypes.c_uint64(int(seed))))

    def sorted_sources(self):
        """(sorted sources (n x 4: x, y, z, m), permutation sorted -> input)."""
        perm = self.arrays()["perm"]
        sp = np.concatenate([self.points[perm], self.masses[perm, None]], axis=1)
        return np.ascontiguousarray(sp, np.float32), perm.astype(np.uint32)

    def plan_stats(self):
        a, b, c = _c_i64(), _c_i64(), _c_i64()
        self._lib.orc_native_plan_stats(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def force(self, eps, cutoff=0.0, points=None, masses=None, w=None, quad=False):
        p = self.points if points is None else _f32(points)
        m = self.masses if masses is None else _f32(masses)
        out = np.zeros((p.shape[0], 3), np.float64)
        loss = ctypes.c_double(0.0)
        ww = _f32(w) if w is not None else None
        self._lib.orc_native_eval(self._h, _ptr(p), _ptr(m), float(eps), float(cutoff), int(quad), _ptr(out), _ptr(ww),
                                  ctypes.byref(loss))
        return out, loss.value

    def finite_differences(self, w, eps, idx, hx=1e-4, hm_rel=1e-4, quad=False):
        """Central FD in float64 of the recorded plan's loss sum_i w_i . a_i
        with respect to the positions (step hx) and masses (step hm_rel * m)
        of the particles idx (orc_native_fd: only the terms each particle
        enters are re-evaluated). Returns (dx (len(idx), 3), dm (len(idx),))."""
        ip = np.ascontiguousarray(np.asarray(idx, np.int64))
        dx = np.zeros((ip.shape[0], 3), np.float64)
        dm = np.zeros(ip.shape[0], np.float64)
        self._lib.orc_native_fd(self._h, _ptr(self.points), _ptr(self.masses), _ptr(_f32(w)), float(eps), int(quad),
                                _ptr(ip), ip.shape[0], float(hx), float(hm_rel), _ptr(dx), _ptr(dm))
        return dx, dm

    def adjoint(self, w, eps, cutoff=0.0, points=None, masses=None, quad=False):
        p = self.points if points is None else _f32(points)
        m = self.masses if masses is None else _f32(masses)
        dx = np.zeros((p.shape[0], 3), np.float64)
        dm = np.zeros(p.shape[0], np.float64)
        self._lib.orc_native_adjoint(self._h, _ptr(p), _ptr(m), _ptr(_f32(w)), float(eps), float(cutoff), int(quad),
                                     _ptr(dx), _ptr(dm))
        return dx, dm


class native_periodic:
    """Context manager: the native plan and sums of the oracle use periodic
    minimum images in a cube of side box and skip cells beyond prune_radius
    of a group (0: no pruning), as the CUDA walk does with those params."""

    def __init__(self, box: float, prune_radius: float = 0.0, periodic: bool = True):
        self.args = (int(bool(periodic)), float(box), float(prune_radius))

    def __enter__(self):
        _orc().orc_native_set_periodic(*self.args)
        return self

    def __exit__(self, *exc):
        _orc().orc_native_set_periodic(0, 1.0, 0.0)
        return False


class native_quadrupole_linear:
    """Context: accepted quadrupole nodes with r_g^2 <= kappa^2 |c - cell centre|^2
    (group box centre c, half diagonal r_g) take the quadrupole to first
    order about c (the CUDA walk's quadrupole_linear); 0 restores the exact
    form everywhere. Plans recorded inside keep their flags."""

    def __init__(self, kappa: float):
        self.kappa = kappa

    def __enter__(self):
        _orc().orc_native_set_quad_linear(self.kappa)
        return self

    def __exit__(self, *exc):
        _orc().orc_native_set_quad_linear(0.0)
        return False


class native_quadrupole_radius:
    """Context manager: plans recorded inside it give an accepted node the
    quadrupole only within q opening radii of the group (q = 0: every
    accepted node), as the CUDA walk does with quadrupole_radius = q."""

    def __init__(self, q: float):
        self.q = float(q)

    def __enter__(self):
        _orc().orc_native_set_quadrupole_radius(self.q)
        return self

    def __exit__(self, *exc):
        _orc().orc_native_set_quadrupole_radius(0.0)
        return False


# ---------------------------------------------------------------------------
# reference CPU code (libsbh_ref_cpu.so / libsbh_ref_cpu64.so)
# ---------------------------------------------------------------------------
REF_K_POTENTIAL, REF_K_WINDING, REF_K_SMOOTHDIST, REF_K_SOFT_FORCE, REF_K_SOFT_FORCE_VJP, REF_K_GRAVITY_GRAD = range(6)


def _refcpu(double: bool = False) -> ctypes.CDLL:
    lib = _load("libsbh_ref_cpu64.so" if double else "libsbh_ref_cpu.so")
    if not getattr(lib, "_typed", False):
        lib.ref_set_softening.argtypes = [_c_d, _c_d]
        lib.ref_tree3d_build.restype = _c_p
        lib.ref_tree3d_build.argtypes = [_c_i, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_f, _c_i]
        lib.ref_tree3d_free.argtypes = [_c_p]
        lib.ref_tree3d_num_nodes.restype = _c_i64
        lib.ref_tree3d_num_nodes.argtypes = [_c_p]
        lib.ref_tree3d_max_depth.restype = _c_i
        lib.ref_tree3d_max_depth.argtypes = [_c_p]
        lib.ref_tree3d_node_size.restype = _c_sz
        lib.ref_tree3d_node_size.argtypes = [_c_i]
        lib.ref_leaf3_size.restype = _c_sz
        lib.ref_leaf2_size.restype = _c_sz
        lib.ref_tree3d_copy_leaf.argtypes = [_c_p, _c_p]
        lib.ref_tree3d_copy_nodes.argtypes = [_c_p, _c_p]
        lib.ref_tree3d_copy_contrib.argtypes = [_c_p, _c_p]
        lib.ref_tree3d_eval.restype = _c_i
        lib.ref_tree3d_eval.argtypes = [_c_p, _c_p, _c_i64, _c_f, _c_i, _c_p, _c_p, _c_p, _c_i]
        lib.ref_tree3d_mlpcv.restype = _c_i
        lib.ref_tree3d_mlpcv.argtypes = [_c_p, _c_p, _c_i64, _c_i, _c_i, _c_u32, _c_p, _c_p, _c_i]
        lib.ref_tree2d_build.restype = _c_p
        lib.ref_tree2d_build.argtypes = [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_f]
        lib.ref_tree2d_free.argtypes = [_c_p]
        lib.ref_tree2d_num_nodes.restype = _c_i64
        lib.ref_tree2d_num_nodes.argtypes = [_c_p]
        lib.ref_tree2d_node_size.restype = _c_sz
        lib.ref_tree2d_copy_leaf.argtypes = [_c_p, _c_p]
        lib.ref_tree2d_copy_nodes.argtypes = [_c_p, _c_p]
        lib.ref_tree2d_copy_contrib.argtypes = [_c_p, _c_p]
        lib.ref_tree2d_eval.restype = _c_i
        lib.ref_tree2d_eval.argtypes = [_c_p, _c_p, _c_i64, _c_f, _c_i, _c_p, _c_p, _c_i]
        lib._typed = True
    return lib


class RefTree3D:
    """The reference's CPU Tree3D (variant 0: <8,1>, 1: <1,1> = Octree1, 2: <1,3> = Octree3)."""

    def __init__(self, points, masses, normals=None, min_corner=None, max_corner=None, variant=0,
                 alpha=1.0, double=False, max_depth=100):
        self.points = _f32(points)
        self.masses = _f32(masses)
        self.normals = _f32(normals) if normals is not None else np.zeros_like(self.points)
        if min_corner is None:
            min_corner = self.points.min(axis=0) - np.float32(1e-3)
        if max_corner is None:
            max_corner = self.points.max(axis=0) + np.float32(1e-3)
        self.min_corner, self.max_corner = _f32(min_corner), _f32(max_corner)
        self.variant = variant
        self._lib = _refcpu(double)
        self._h = self._lib.ref_tree3d_build(variant, _ptr(self.points), _ptr(self.normals), _ptr(self.masses),
                                             self.points.shape[0], _ptr(self.min_corner), _ptr(self.max_corner),
                                             float(alpha), int(max_depth))

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ref_tree3d_free(self._h)
            self._h = None

    @property
    def num_nodes(self) -> int:
        return int(self._lib.ref_tree3d_num_nodes(self._h))

    def leaf_bytes(self) -> np.ndarray:
        out = np.zeros(self.points.shape[0] * int(self._lib.ref_leaf3_size()), np.uint8)
        self._lib.ref_tree3d_copy_leaf(self._h, _ptr(out))
        return out

    def node_bytes(self) -> np.ndarray:
        out = np.zeros(self.num_nodes * int(self._lib.ref_tree3d_node_size(self.variant)), np.uint8)
        self._lib.ref_tree3d_copy_nodes(self._h, _ptr(out))
        return out

    def contrib_bytes(self) -> np.ndarray:
        out = np.zeros(self.num_nodes * int(self._lib.ref_leaf3_size()), np.uint8)
        self._lib.ref_tree3d_copy_contrib(self._h, _ptr(out))
        return out

    def eval(self, queries, beta, kernel, eps=1e-3, cutoff=0.0, cot=None, threads=0):
        q = _f32(queries)
        vec = kernel in (REF_K_SOFT_FORCE, REF_K_SOFT_FORCE_VJP, REF_K_GRAVITY_GRAD)
        out = np.zeros((q.shape[0], 3) if vec else q.shape[0], np.float64)
        counts = np.zeros(q.shape[0], np.int32)
        self._lib.ref_set_softening(float(eps), float(cutoff))
        g = _f32(cot) if cot is not None else None
        self._lib.ref_tree3d_eval(self._h, _ptr(q), q.shape[0], float(beta), int(kernel), _ptr(g), _ptr(out),
                                  _ptr(counts), int(threads))
        return out, counts

    def mlpcv(self, queries, kernel, samples, seed, eps=1e-3, cutoff=0.0, threads=0):
        q = _f32(queries)
        vec = kernel in (REF_K_SOFT_FORCE, REF_K_GRAVITY_GRAD)
        out = np.zeros((q.shape[0], 3) if vec else q.shape[0], np.float64)
        counts = np.zeros(q.shape[0], np.int32)
        self._lib.ref_set_softening(float(eps), float(cutoff))
        self._lib.ref_tree3d_mlpcv(self._h, _ptr(q), q.shape[0], int(kernel), int(samples), int(seed) & 0xFFFFFFFF,
                                   _ptr(out), _ptr(counts), int(threads))
        return out, counts


class RefTree2D:
    """The reference's CPU Tree2D<1,3> (sbh.Quadtree3): the Node2 layout builder."""

    def __init__(self, points, masses, normals=None, min_corner=None, max_corner=None, alpha=1.0):
        self.points = _f32(points)
        self.masses = _f32(masses)
        self.normals = _f32(normals) if normals is not None else np.zeros_like(self.points)
        if min_corner is None:
            min_corner = self.points.min(axis=0) - np.float32(1e-3)
        if max_corner is None:
            max_corner = self.points.max(axis=0) + np.float32(1e-3)
        self._lib = _refcpu(False)
        self._h = self._lib.ref_tree2d_build(_ptr(self.points), _ptr(self.normals), _ptr(self.masses),
                                             self.points.shape[0], _ptr(_f32(min_corner)), _ptr(_f32(max_corner)),
                                             float(alpha))

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ref_tree2d_free(self._h)
            self._h = None

    @property
    def num_nodes(self) -> int:
        return int(self._lib.ref_tree2d_num_nodes(self._h))

    def leaf_bytes(self):
        out = np.zeros(self.points.shape[0] * int(self._lib.ref_leaf2_size()), np.uint8)
        self._lib.ref_tree2d_copy_leaf(self._h, _ptr(out))
        return out

    def node_bytes(self):
        out = np.zeros(self.num_nodes * int(self._lib.ref_tree2d_node_size()), np.uint8)
        self._lib.ref_tree2d_copy_nodes(self._h, _ptr(out))
        return out

    def contrib_bytes(self):
        out = np.zeros(self.num_nodes * int(self._lib.ref_leaf2_size()), np.uint8)
        self._lib.ref_tree2d_copy_contrib(self._h, _ptr(out))
        return out

    def eval(self, queries, beta, kernel, threads=0):
        q = _f32(queries)
        vec = kernel == REF_K_GRAVITY_GRAD
        out = np.zeros((q.shape[0], 2) if vec else q.shape[0], np.float64)
        counts = np.zeros(q.shape[0], np.int32)
        self._lib.ref_tree2d_eval(self._h, _ptr(q), q.shape[0], float(beta), int(kernel), _ptr(out), _ptr(counts),
                                  int(threads))
        return out, counts


# ---------------------------------------------------------------------------
# reference GPU plugin (libsbh_ref_gpu.so); pointers are device addresses
# ---------------------------------------------------------------------------
def refgpu() -> ctypes.CDLL:
    """The reference's src/sbh_ffi.cu handlers behind extern "C" wrappers."""
    lib = _load("libsbh_ref_gpu.so")
    if not getattr(lib, "_typed", False):
        lib.ref_gpu_last_error.restype = ctypes.c_char_p
        for nm in ("ref_gpu_leaf3_size", "ref_gpu_node3_size", "ref_gpu_octree8_node_size", "ref_gpu_level3_max_nodes"):
            getattr(lib, nm).restype = _c_sz
        lib.ref_bruteforce_gravity.argtypes = [_c_p, _c_p, _c_p, _c_i64, _c_i, _c_p, _c_i64, _c_p, _c_i, _c_f, _c_i]
        lib.ref_sbhgpu_barnes_hut.argtypes = [_c_p, _c_i, _c_i, _c_p, _c_p, _c_p, _c_i64, _c_f, _c_p]
        lib.ref_sbhgpu_mlpcv.argtypes = [_c_p, _c_i, _c_i, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_i64, _c_i, _c_p]
        lib.ref_sbhgpu_brute.argtypes = [_c_p, _c_i, _c_i, _c_p, _c_i64, _c_p, _c_i64, _c_p]
        lib.ref_direct_force_soft.argtypes = [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_f, _c_f, _c_i, _c_f, _c_i]
        lib.ref_direct_force_soft_vjp.argtypes = [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_p, _c_f, _c_f, _c_i,
                                                  _c_f, _c_i]
        lib.ref_build_octree_level3.argtypes = [_c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_i64,
                                                _c_p, _c_i64]
        lib.ref_build_octree8.argtypes = [_c_p, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p,
                                          _c_i64, _c_i]
        lib.ref_barnes_hut_gravity.argtypes = [_c_p, _c_i, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_f, _c_i,
                                               _c_f, _c_i]
        lib.ref_barnes_hut_force.argtypes = lib.ref_barnes_hut_gravity.argtypes
        lib.ref_barnes_hut_force_soft.argtypes = [_c_p, _c_i, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_f,
                                                  _c_f, _c_f, _c_i, _c_f, _c_i]
        lib.ref_stochastic_bh_gravity.argtypes = [_c_p, _c_i, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64,
                                                  _c_p, _c_i, _c_i, _c_i, _c_f, _c_i]
        lib.ref_stochastic_bh_force.argtypes = lib.ref_stochastic_bh_gravity.argtypes
        lib.ref_stochastic_bh_force_soft.argtypes = [_c_p, _c_i, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p,
                                                     _c_i64, _c_p, _c_i, _c_i, _c_f, _c_f, _c_i, _c_f, _c_i]
        lib.ref_bh_force_octree8.argtypes = [_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_f, _c_i, _c_f, _c_i]
        lib.ref_bh_force_octree8_soft.argtypes = [_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_f, _c_f,
                                                  _c_f, _c_i, _c_f, _c_i, _c_f, _c_i]
        lib.ref_bh_force_octree8_soft_vjp.argtypes = [_c_p, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_p, _c_f,
                                                      _c_f, _c_f, _c_i, _c_f, _c_i, _c_f, _c_i]
        lib.ref_stochastic_bh_force_octree8.argtypes = [_c_p, _c_i, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p,
                                                        _c_i, _c_i, _c_f, _c_f, _c_f, _c_i, _c_f, _c_i, _c_f, _c_i]
        lib.ref_stochastic_bh_force_octree8_vjp.argtypes = [_c_p, _c_i, _c_p, _c_i64, _c_p, _c_i64, _c_p, _c_i64, _c_p,
                                                            _c_p, _c_i, _c_i, _c_f, _c_f, _c_f, _c_i, _c_f, _c_i, _c_f,
                                                            _c_i]
        for nm in ("ref_bruteforce_gravity", "ref_direct_force_soft", "ref_direct_force_soft_vjp",
                   "ref_build_octree_level3", "ref_build_octree8", "ref_barnes_hut_gravity", "ref_barnes_hut_force",
                   "ref_barnes_hut_force_soft", "ref_stochastic_bh_gravity", "ref_stochastic_bh_force",
                   "ref_stochastic_bh_force_soft", "ref_bh_force_octree8", "ref_bh_force_octree8_soft",
                   "ref_bh_force_octree8_soft_vjp", "ref_stochastic_bh_force_octree8",
                   "ref_stochastic_bh_force_octree8_vjp"):
            getattr(lib, nm).restype = _c_i
        lib._typed = True
    return lib


def refgpu_check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("reference handler failed: " + refgpu().ref_gpu_last_error().decode())


# ---------------------------------------------------------------------------
# mesh surface sampling (pure numpy restatement of sbh_sample_mesh_surface)
# ---------------------------------------------------------------------------
_SPLITMIX_GAMMA = np.uint64(0x9E3779B97F4A7C15)


def splitmix64_mix(z: np.ndarray) -> np.ndarray:
    """The splitmix64 output function (S. Vigna, 2015) on uint64 arrays; the
    generator's k-th output from seed s is splitmix64_mix(s + k * gamma)."""
    z = np.asarray(z, dtype=np.uint64)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def mesh_face_geometry(V, F):
    """(twice the face areas (float64), unit normals (float32)) in the order
    of operations of the sampler's face pass: e1 = v1 - v0, e2 = v2 - v0 and
    c = e1 x e2 in float64 from the float32 vertices, |c| =
    sqrt((c0^2 + c1^2) + c2^2), normal = c / |c| rounded to float32.
    Degenerate and NaN faces get zero area and a zero normal (the reference
    zeroes NaN areas, python/old_interface/sampler.py:67-68)."""
    V = np.asarray(V, dtype=np.float32).astype(np.float64)
    F = np.asarray(F, dtype=np.int64)
    v0, v1, v2 = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    e1, e2 = v1 - v0, v2 - v0
    c = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1],
                  e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                  e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], axis=1)
    with np.errstate(invalid="ignore"):
        ln = np.sqrt((c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1]) + c[:, 2] * c[:, 2])
    ok = (ln > 0) & np.isfinite(ln)
    ln = np.where(ok, ln, 0.0)
    nrm = np.zeros_like(c)
    nrm[ok] = c[ok] / ln[ok, None]
    return ln, nrm.astype(np.float32)


def sample_points_on_mesh(num_particles: int, V, F, seed: int = 0):
    """Restatement of sbh_sample_mesh_surface (same distribution as the
    reference's sample_points_on_mesh, python/old_interface/sampler.py:63-78):
    sample i draws u0, u1, u2 = outputs 3i+1, 3i+2, 3i+3 of splitmix64 seeded
    with `seed` (top 53 bits / 2^53); its face is the first face whose
    cumulative doubled area exceeds min(u0 * total, the double below total);
    (u1, u2) is reflected to (1 - u1, 1 - u2) when u1 + u2 > 1; the point is
    (v0 + u1 e1) + u2 e2 in float64 rounded to float32; its normal the face's
    unit normal; its weight (total / 2) / n as float32. Returns (points,
    normals, weights, faces)."""
    n = int(num_particles)
    V64 = np.asarray(V, dtype=np.float32).astype(np.float64)
    F = np.asarray(F, dtype=np.int64)
    area2, nrm = mesh_face_geometry(V, F)
    cdf = np.concatenate([[0.0], np.cumsum(area2)])
    total = cdf[-1]
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):  # uint64 arithmetic wraps modulo 2^64, as on the device
        base = np.uint64(seed) + (np.uint64(3) * i + np.uint64(1)) * _SPLITMIX_GAMMA
        u = [(splitmix64_mix(base + np.full(n, k, np.uint64) * _SPLITMIX_GAMMA) >> np.uint64(11)).astype(np.float64)
             * 2.0 ** -53 for k in range(3)]
    top = np.nextafter(total, 0.0)
    target = np.minimum(u[0] * total, top)
    face = np.searchsorted(cdf[1:], target, side="right")
    u1, u2 = u[1], u[2]
    flip = (u1 + u2) > 1.0
    u1 = np.where(flip, 1.0 - u1, u1)
    u2 = np.where(flip, 1.0 - u2, u2)
    v0 = V64[F[face, 0]]
    e1 = V64[F[face, 1]] - v0
    e2 = V64[F[face, 2]] - v0
    pts = ((v0 + u1[:, None] * e1) + u2[:, None] * e2).astype(np.float32)
    w = np.full(n, np.float32((total * 0.5) / n) if n else 0.0, dtype=np.float32)
    return pts, nrm[face], w, face


def mesh_vertex_sources(V, F):
    """Restatement of sbh_mesh_vertex_sources (the reference's MeshVertices,
    python/old_interface/source.py:85-115, whose libigl calls are
    per_vertex_normals(V, F, 1) and the diagonal of massmatrix): per vertex,
    the normalised sum of c = (v1 - v0) x (v2 - v0) over its faces (area
    weighting), and the mixed Voronoi area of Meyer, Desbrun, Schroeder and
    Barr (2003) summed over its faces. Per face with corner angles theta_i:
    without an obtuse angle, corner i takes (|Pi Pk|^2 cot theta_j +
    |Pi Pj|^2 cot theta_k) / 8; with one at corner i, corner i takes area / 2
    and the others area / 4. float64 from the float32 vertices, faces of zero
    area skipped; returns (normals float64, masses float64)."""
    V = np.asarray(V, dtype=np.float32).astype(np.float64)
    F = np.asarray(F, dtype=np.int64)
    nv = V.shape[0]
    P = [V[F[:, c]] for c in range(3)]
    e = [P[(c + 1) % 3] - P[c] for c in range(3)]  # edge from corner c to c + 1
    n = np.cross(e[0], P[2] - P[0])
    dbl = np.linalg.norm(n, axis=1)
    ok = (dbl > 0) & np.isfinite(dbl)
    F, n, dbl = F[ok], n[ok], dbl[ok]
    e = [x[ok] for x in e]
    area = 0.5 * dbl
    l2 = [np.einsum("ij,ij->i", x, x) for x in e]
    dot = [-np.einsum("ij,ij->i", e[c], e[(c + 2) % 3]) for c in range(3)]  # corner c: P(c+1)-Pc . P(c-1)-Pc
    cot = [d / dbl for d in dot]
    share = np.stack([(l2[c] * cot[(c + 2) % 3] + l2[(c + 2) % 3] * cot[(c + 1) % 3]) / 8.0 for c in range(3)],
                     axis=1)
    for c in range(3):
        ob = dot[c] < 0
        share[ob] = 0.25 * area[ob, None]
        share[ob, c] = 0.5 * area[ob]
    mass = np.zeros(nv)
    nsum = np.zeros((nv, 3))
    for c in range(3):
        np.add.at(mass, F[:, c], share[:, c])
        np.add.at(nsum, F[:, c], n)
    ln = np.linalg.norm(nsum, axis=1)
    nrm = np.zeros_like(nsum)
    good = ln > 0
    nrm[good] = nsum[good] / ln[good, None]
    return nrm, mass


def native_stochastic(sorted_sources, perm, node_records, *, group_size=128, beta_coarse=1.0, beta=2.0,
                      softening=1e-3, samples=32, seed=0, expectation=True):
    """The native stochastic Barnes-Hut estimator restated (orc_native_stochastic)
    on given node records (the GPU export, or NativeTree.node_records()).
    Returns (estimate, expectation or None, subtree walks), the first two
    float64 n x 3 in input order. softening enters as eps^2 + 1e-12 in
    float, as the CUDA walk holds it."""
    sp = _f32(sorted_sources)
    pm = np.ascontiguousarray(np.asarray(perm, np.uint32))
    nodes = np.ascontiguousarray(np.asarray(node_records, np.uint8))
    n, nn = sp.shape[0], nodes.size // 80
    eps2 = np.float32(np.float32(softening) * np.float32(softening) + np.float32(1e-12))
    out = np.zeros((n, 3), np.float64)
    ex = np.zeros((n, 3), np.float64) if expectation else None
    walks = _orc().orc_native_stochastic(_ptr(sp), _ptr(pm), n, _ptr(nodes), nn, int(group_size), float(beta_coarse),
                                         float(beta), float(eps2), int(samples), ctypes.c_uint64(int(seed)),
                                         _ptr(out), _ptr(ex))
    return out, ex, int(walks)
