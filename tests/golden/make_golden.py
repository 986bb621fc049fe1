"""Generate golden fixtures from the REFERENCE's own GPU plugin.

Runs the reference's src/sbh_ffi.cu handlers (compiled unmodified into
oracle/_ref/libsbh_ref_gpu.so by `make -C oracle ref`) on small seeded
inputs and stores inputs and outputs as .npz files. Needs a CUDA device; run
it on the GPU box and commit the resulting files under tests/golden/:

    python tests/golden/make_golden.py <out_dir>

The fixtures pin the CPU oracle (tests/test_golden.py) and the library's
kernels (tests/test_gpu_compat.py) to the reference's outputs.
"""
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "barnes-hut_b200"))
import sbh_oracle as O  # noqa: E402
import sbh_workloads as W  # noqa: E402

DEV = torch.device("cuda", 0)


def t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), device=DEV, dtype=dtype)


def S():
    return torch.cuda.current_stream().cuda_stream


def ref_build_octree8(p, nrm, m, mn, mx, depth):
    L = O.refgpu()
    n = p.shape[0]
    total = O.octree8_total_nodes(depth)
    leaf = torch.zeros(n * 32, dtype=torch.uint8, device=DEV)
    node = torch.zeros(total * 104, dtype=torch.uint8, device=DEV)
    contrib = torch.zeros(total * 32, dtype=torch.uint8, device=DEV)
    P, N, M, MN, MX = t(p), t(nrm), t(m), t(mn), t(mx)
    O.refgpu_check(L.ref_build_octree8(S(), P.data_ptr(), N.data_ptr(), M.data_ptr(), n, MN.data_ptr(), MX.data_ptr(),
                                       leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                       contrib.data_ptr(), contrib.numel(), depth))
    torch.cuda.synchronize()
    return leaf, node, contrib


def octree8_fixture(out_dir):
    rng = np.random.default_rng(101)
    cases = {}
    pu, mu = W.uniform_cube(1500, seed=12)
    pp, mp = W.plummer(2048, seed=11)
    pp = pp * np.float32(0.2)
    cases["uniform"] = (pu, mu)
    cases["plummer"] = (pp, mp)
    res = {}
    L = O.refgpu()
    for name, (p, m) in cases.items():
        nrm = rng.normal(size=p.shape).astype(np.float32)
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        mn = (p.min(0) - np.float32(1e-3)).astype(np.float32)
        mx = (p.max(0) + np.float32(1e-3)).astype(np.float32)
        for depth in (3, 5):
            leaf, node, contrib = ref_build_octree8(p, nrm, m, mn, mx, depth)
            key = f"{name}_d{depth}"
            res[key + "_points"] = p
            res[key + "_normals"] = nrm
            res[key + "_masses"] = m
            res[key + "_min"] = mn
            res[key + "_max"] = mx
            res[key + "_leaf"] = leaf.cpu().numpy()
            res[key + "_node"] = node.cpu().numpy()
            res[key + "_contrib"] = contrib.cpu().numpy()
            if depth != 5:
                continue
            q = np.concatenate([p[:256], rng.uniform(p.min(0), p.max(0), (64, 3)).astype(np.float32)])
            cot = rng.normal(size=q.shape).astype(np.float32)
            Q, C = t(q), t(cot)
            res[key + "_queries"] = q
            res[key + "_cot"] = cot
            nq = q.shape[0]

            def run(fn, args):
                out = torch.zeros((nq, 3), dtype=torch.float32, device=DEV)
                O.refgpu_check(fn(S(), *args(out)))
                torch.cuda.synchronize()
                return out.cpu().numpy()

            lb, nb = leaf.numel(), node.numel()
            lp, np_ = leaf.data_ptr(), node.data_ptr()
            res[key + "_bh_beta2"] = run(L.ref_bh_force_octree8,
                                         lambda o: (lp, lb, np_, nb, Q.data_ptr(), nq, o.data_ptr(), 2.0, 0, 1.0, 256))
            for tag, (eps, cut, prune, mult) in {"soft": (5e-2, 1.5, 0, 4.0), "softprune": (5e-2, 0.3, 1, 2.0),
                                                 "plummer": (1e-3, 1e6, 1, 4.0)}.items():
                res[key + f"_{tag}"] = run(L.ref_bh_force_octree8_soft,
                                           lambda o: (lp, lb, np_, nb, Q.data_ptr(), nq, o.data_ptr(), 2.0, eps, cut,
                                                      prune, mult, 0, 1.0, 256))
                res[key + f"_{tag}_vjp"] = run(L.ref_bh_force_octree8_soft_vjp,
                                               lambda o: (lp, lb, np_, nb, Q.data_ptr(), nq, C.data_ptr(), o.data_ptr(),
                                                          2.0, eps, cut, prune, mult, 0, 1.0, 256))
            for seed in (7, 11):
                for soft in (0, 1):
                    res[key + f"_stoch_s{seed}_soft{soft}"] = run(
                        L.ref_stochastic_bh_force_octree8,
                        lambda o: (soft, lp, lb, np_, nb, Q.data_ptr(), nq, o.data_ptr(), 2, seed, 1.0, 5e-2, 1.5, 1,
                                   4.0, 0, 1.0, 256))
                    res[key + f"_stoch_s{seed}_soft{soft}_vjp"] = run(
                        L.ref_stochastic_bh_force_octree8_vjp,
                        lambda o: (soft, lp, lb, np_, nb, Q.data_ptr(), nq, C.data_ptr(), o.data_ptr(), 2, seed, 1.0,
                                   5e-2, 1.5, 1, 4.0, 0, 1.0, 256))
    # periodic case (test_jax_ffi_tree_builder.py:264-305 shapes)
    box = 2.0
    p = rng.uniform(0, box, (192, 3)).astype(np.float32)
    m = np.ones(192, np.float32)
    mn = np.zeros(3, np.float32)
    mx = np.full(3, box, np.float32)
    leaf, node, contrib = ref_build_octree8(p, np.zeros_like(p), m, mn, mx, 5)
    q = p[:32]
    Q = t(q)
    out = torch.zeros((32, 3), dtype=torch.float32, device=DEV)
    O.refgpu_check(L.ref_bh_force_octree8(S(), leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                          Q.data_ptr(), 32, out.data_ptr(), 1.8, 1, box, 256))
    torch.cuda.synchronize()
    res.update(periodic_points=p, periodic_leaf=leaf.cpu().numpy(), periodic_node=node.cpu().numpy(),
               periodic_force=out.cpu().numpy())
    np.savez_compressed(os.path.join(out_dir, "octree8_reference.npz"), **res)


def direct_fixture(out_dir):
    L = O.refgpu()
    rng = np.random.default_rng(23)
    p = rng.uniform(-1, 1, (96, 3)).astype(np.float32)
    m = rng.uniform(0.1, 1.3, 96).astype(np.float32)
    q = rng.uniform(-0.7, 0.7, (31, 3)).astype(np.float32)
    g = rng.normal(size=(31, 3)).astype(np.float32)
    P, M, Q, G = t(p), t(m), t(q), t(g)
    f = torch.zeros((31, 3), device=DEV)
    v = torch.zeros((31, 3), device=DEV)
    O.refgpu_check(L.ref_direct_force_soft(S(), P.data_ptr(), M.data_ptr(), 96, Q.data_ptr(), 31, f.data_ptr(), 5e-2,
                                           0.9, 0, 1.0, 256))
    O.refgpu_check(L.ref_direct_force_soft_vjp(S(), P.data_ptr(), M.data_ptr(), 96, Q.data_ptr(), 31, G.data_ptr(),
                                               v.data_ptr(), 7e-2, 1.4, 0, 1.0, 256))
    res = dict(points=p, masses=m, queries=q, cot=g, force=f.cpu().numpy(), vjp=v.cpu().numpy())
    for dim in (2, 3):
        pd = rng.uniform(-1, 1, (80, dim)).astype(np.float32)
        qd = rng.uniform(-1, 1, (40, dim)).astype(np.float32)
        md = rng.uniform(0.1, 1, 80).astype(np.float32)
        out = torch.zeros(40, device=DEV)
        PD, MD, QD = t(pd), t(md), t(qd)
        O.refgpu_check(L.ref_bruteforce_gravity(S(), PD.data_ptr(), MD.data_ptr(), 80, dim, QD.data_ptr(), 40,
                                                out.data_ptr(), 0, 1.0, 64))
        res.update({f"bf{dim}_points": pd, f"bf{dim}_masses": md, f"bf{dim}_queries": qd,
                    f"bf{dim}_out": out.cpu().numpy()})
    torch.cuda.synchronize()
    np.savez_compressed(os.path.join(out_dir, "direct_reference.npz"), **res)


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    os.makedirs(out_dir, exist_ok=True)
    direct_fixture(out_dir)
    octree8_fixture(out_dir)
    print("golden fixtures written to", out_dir)


if __name__ == "__main__":
    main()
